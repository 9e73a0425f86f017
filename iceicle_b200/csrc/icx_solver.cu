// Newton solver around the GPU residual and FD Jacobian:
//   PetscNewton::solve (src/solvers/include/iceicle/petsc_newton.hpp:205-329)
//   with the reference's line searches (nonlinear_solver_utils.hpp:83-191)
// and the linear solve J du = r by restarted, right-preconditioned GMRES(m)
// (classical Gram-Schmidt with one re-orthogonalisation, FP64 Hessenberg and
// Givens rotations on the host) with block-Jacobi or block-ILU(0)
// preconditioning on the BSR Jacobian. Every vector operation runs on the
// device; the host holds only the (m+1) x m Hessenberg matrix and the scalar
// line-search logic.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <vector>

#include "icx_internal.h"
#include "icx_linalg.h"

// block-ILU(0) on s x s element tiles (icx_ctx::ilu_tile = s > 0): the
// preconditioner keeps only the blocks that couple two elements of the same
// tile, i.e. block-Jacobi over the tiles with ILU(0) inside each (the form of
// PETSc's parallel default, bjacobi with ilu sub-solves, with one block per
// tile). On a quadrilateral grid no ILU(0) update couples two face
// neighbours, so dropping the cross-tile blocks leaves every in-tile factor
// block exactly what ILU(0) of the tile's own matrix gives. The dependent
// levels of the factorisation and of each triangular sweep fall from
// nx + ny - 1 to 2s - 1.
struct IluTilePlan {
  int tile = 0;                 // nonzero: a plan is built (s, or -1 for element groups)
  int gen = 0;                  // icx_ctx::ilu_plan_gen it was built for
  int nnzb = 0;                 // blocks kept
  int* rowptr = nullptr;        // [E + 1] kept pattern, columns ascending
  int* colidx = nullptr;        // [nnzb]
  int* diag = nullptr;          // [E] position of the diagonal block
  int* map = nullptr;           // [nnzb] kept block -> block of the full pattern
  int* order = nullptr;         // [E] elements by ascending in-tile level (i mod s) + (j mod s)
  std::vector<int> lvl_off;
  // the same per group (one CTA per group, la_ilu_apply_groups): elements
  // group by group, by level within the group, and each group's level bounds
  int ngroups = 0;
  int gmax = 0;                 // elements of the largest group
  int nlev_max = 0;             // most levels of a group
  bool group_ok = true;         // no sweep row has more than two off-diagonal blocks
  int* gtask = nullptr;         // [2 E] x 4: IluGroupPlan::task, in group order (group, level, element)
  int* gloc = nullptr;          // [2 E] x 4: IluGroupPlan::loc
  int* glev = nullptr;          // level boundaries (positions in the group order), per group
  int* glev_ptr = nullptr;      // [ngroups + 1] into glev
};

struct icx_solver_work {
  long long n = 0;
  int nnzb = 0, bs = 0, m = 0;
  double* vals = nullptr;   // Jacobian
  double* pc = nullptr;     // preconditioner: block inverses (Jacobi) or ILU factors
  double* uinv = nullptr;   // ILU: inverses of the U diagonal blocks
  double* V = nullptr;      // Krylov basis, (m + 1) x n
  double* w = nullptr;      // work vectors
  double* z = nullptr;
  double* r = nullptr;      // GMRES restart residual (internal to gmres)
  double* res = nullptr;    // Newton residual R(u), the right-hand side of the linear solves
  double* du = nullptr;
  double* ustep = nullptr;
  double* rwork = nullptr;
  double* pct = nullptr;    // scratch of the preconditioner apply
  double* pct2 = nullptr;
  double* pct3 = nullptr;
  double* pct4 = nullptr;
  int sweeps = 2;           // Jacobi sweeps per triangle (preconditioner 4)
  float* vals32 = nullptr;  // mixed precision: FP32 copies of the Jacobian and the preconditioner
  float* pc32 = nullptr;
  float* uinv32 = nullptr;
  // BF16 copies of the ILU factors (Newton precision 3: the tiled apply's
  // one-lane-per-row form reads them, widening to FP32)
  bool bf16 = false;
  __nv_bfloat16* pc16 = nullptr;
  __nv_bfloat16* uinv16 = nullptr;
  float* V32 = nullptr;     // mixed precision: the Krylov basis in FP32, (m + 1) x n
  double* vt = nullptr;     // the basis vector widened for the operators
  int* order = nullptr;     // elements by ascending level (ILU schedule)
  std::vector<int> lvl_off; // level l: order[lvl_off[l] .. lvl_off[l+1])
  unsigned* cnt = nullptr;  // 2 x E completion counters of the ILU apply
  unsigned epoch = 0;       // ILU applies since the counters were zeroed
  // rows per task of those applies: an element's counter grows by its task
  // count per apply (block size / rows), so the counters restart when it changes
  int flow_rows = 0;
  icx::ArnoldiGraphs graphs;  // CUDA graphs of the GMRES Arnoldi steps
  bool graphs_on = true;      // use them where the preconditioner allows (icx_newton_options.cuda_graphs)
  long long graph_steps = 0;  // Arnoldi steps replayed from them
  // row-pipelined ILU apply: the context is one structured grid whose block
  // pattern is the 5-point element stencil in natural order
  bool rows_ok = false;
  int schedule = 0;         // 0 / 1: data flow (the solvers' apply), 2: rows (icx_ilu_apply only)
  unsigned* cnt_rows = nullptr;
  unsigned epoch_rows = 0;
  IluTilePlan tp;           // tiled block-ILU(0) pattern and schedule (tp.tile == c->ilu_tile once built)
  int* pc_err = nullptr;    // set by the ILU apply if a dependency wait timed out
  double* dh = nullptr;     // device scalars (dot results)
  // the matrix-free operator (icx_newton_options.matrix_free) while a Newton
  // step's linear solve runs: state, its residual, {|v|^2, c} (in dh)
  int cgs_passes = 2;       // Gram-Schmidt passes of the GMRES run by a Newton step
  bool fd_on = false;
  const double* fd_u = nullptr;
  const double* fd_r = nullptr;
  double* fd_slot = nullptr;
  int* flag = nullptr;
  icx::LinalgWork lw;
};

namespace {

icx_status set_err(icx_ctx* c, icx_status st, const std::string& m) {
  if (c) c->err = m;
  return st;
}

// synchronises and reports any failure of the work enqueued so far, tagged
#define SYNC_AT(tag)                                                                            \
  do {                                                                                          \
    cudaError_t _e = cudaStreamSynchronize(s);                                                  \
    if (_e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string(tag) + ": " + cudaGetErrorString(_e)); \
  } while (0)

#define CK(expr)                                                                       \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string(#expr) + ": " + \
                                                              cudaGetErrorString(_e)); \
  } while (0)

icx_status ensure_work(icx_ctx* c, int m) {
  const icx::DeviceMesh& dm = c->dm;
  long long n = (long long)dm.E * dm.nb * dm.neq;
  int bs = dm.nb * dm.neq;
  icx_solver_work*& w = c->sw;
  if (w && w->n == n && w->nnzb == dm.nnzb && w->bs == bs && w->m >= m) return ICX_OK;
  icx::free_solver_work(c);
  w = new icx_solver_work();
  w->n = n;
  w->nnzb = dm.nnzb;
  w->bs = bs;
  w->m = m;
  size_t vb = sizeof(double) * (size_t)dm.nnzb * bs * bs;
  CK(cudaMalloc((void**)&w->vals, vb));
  CK(cudaMalloc((void**)&w->pc, vb));
  CK(cudaMalloc((void**)&w->uinv, sizeof(double) * (size_t)dm.E * bs * bs));
  CK(cudaMalloc((void**)&w->V, sizeof(double) * (size_t)(m + 1) * n));
  double** vecs[] = {&w->w, &w->z, &w->r, &w->res, &w->du, &w->ustep, &w->rwork, &w->pct, &w->pct2, &w->pct3, &w->pct4};
  for (double** p : vecs) CK(cudaMalloc((void**)p, sizeof(double) * n));
  // 3 (m + 2) GMRES reductions, then the matrix-free products' {|v|^2, c}
  CK(cudaMalloc((void**)&w->dh, sizeof(double) * (3 * (m + 2) + 2)));
  CK(cudaMalloc((void**)&w->flag, sizeof(int)));
  CK(cudaMalloc((void**)&w->pc_err, sizeof(int)));
  CK(cudaMemset(w->pc_err, 0, sizeof(int)));
  CK(cudaMalloc((void**)&w->cnt, sizeof(unsigned) * 2 * dm.E));
  CK(cudaMemset(w->cnt, 0, sizeof(unsigned) * 2 * dm.E));
  {
    // elements by ascending level (anti-diagonal of the element in its grid)
    int nl = 0;
    for (int v : c->el_level) nl = std::max(nl, v + 1);
    w->lvl_off.assign(nl + 1, 0);
    for (int v : c->el_level) ++w->lvl_off[v + 1];
    for (int l = 0; l < nl; ++l) w->lvl_off[l + 1] += w->lvl_off[l];
    std::vector<int> order(dm.E), fill(w->lvl_off.begin(), w->lvl_off.end() - 1);
    for (int e = 0; e < dm.E; ++e) order[fill[c->el_level[e]]++] = e;
    CK(cudaMalloc((void**)&w->order, sizeof(int) * dm.E));
    CK(cudaMemcpy(w->order, order.data(), sizeof(int) * dm.E, cudaMemcpyHostToDevice));
  }
  CK(cudaMalloc((void**)&w->lw.partial, sizeof(double) * 64 * icx::kMdotBlocks));
  CK(cudaMalloc((void**)&w->cnt_rows, sizeof(unsigned) * 2 * dm.E));
  CK(cudaMemset(w->cnt_rows, 0, sizeof(unsigned) * 2 * dm.E));
  if (c->parts.empty() && c->nx > 0 && c->ny > 0 && (long long)c->nx * c->ny == dm.E) {
    // the 5-point element stencil in natural order: row e holds e-nx, e-1, e, e+1, e+nx where they exist
    std::vector<int> rp(dm.E + 1), ci(dm.nnzb);
    CK(cudaMemcpy(rp.data(), dm.bsr_rowptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ci.data(), dm.bsr_colidx, sizeof(int) * ci.size(), cudaMemcpyDeviceToHost));
    bool ok = true;
    const int nx = c->nx, ny = c->ny;
    for (int e = 0; e < dm.E && ok; ++e) {
      const int i = e % nx, j = e / nx;
      std::vector<int> want;
      if (j > 0) want.push_back(e - nx);
      if (i > 0) want.push_back(e - 1);
      want.push_back(e);
      if (i < nx - 1) want.push_back(e + 1);
      if (j < ny - 1) want.push_back(e + nx);
      ok = (rp[e + 1] - rp[e]) == (int)want.size();
      for (size_t k = 0; ok && k < want.size(); ++k) ok = ci[rp[e] + k] == want[k];
    }
    w->rows_ok = ok;
  }
  return ICX_OK;
}

void free_tile_plan(IluTilePlan& tp) {
  for (int* p : {tp.rowptr, tp.colidx, tp.diag, tp.map, tp.order, tp.gtask, tp.gloc, tp.glev, tp.glev_ptr})
    if (p) cudaFree(p);
  tp = IluTilePlan();
}

// builds the pattern of the tiled (c->ilu_tile) or grouped (c->ilu_groups)
// block-ILU(0); nothing to do when it is built or when neither is set
icx_status ensure_ilu_plan(icx_ctx* c) {
  icx_solver_work* w = c->sw;
  const bool grouped = !c->ilu_groups.empty();
  const int st = grouped ? -1 : c->ilu_tile;
  if (st == w->tp.tile && (st == 0 || w->tp.gen == c->ilu_plan_gen)) return ICX_OK;
  free_tile_plan(w->tp);
  if (st == 0) return ICX_OK;
  const icx::DeviceMesh& dm = c->dm;
  if (grouped && (int)c->ilu_groups.size() != dm.E)
    return set_err(c, ICX_ERR_INVALID, "ILU element groups: one group per element");
  if (!grouped && ((int)c->el_i.size() != dm.E || (int)c->el_j.size() != dm.E || (int)c->el_grid.size() != dm.E))
    return set_err(c, ICX_ERR_UNSUPPORTED, "tiled block-ILU(0) needs the elements' grid positions");
  std::vector<int> rp(dm.E + 1), ci(dm.nnzb);
  CK(cudaMemcpy(rp.data(), dm.bsr_rowptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ci.data(), dm.bsr_colidx, sizeof(int) * ci.size(), cudaMemcpyDeviceToHost));
  auto tile_of = [&](int e) -> long long {
    if (grouped) return c->ilu_groups[e];
    return ((long long)c->el_grid[e] << 42) | ((long long)(c->el_i[e] / st) << 21) | (long long)(c->el_j[e] / st);
  };
  std::vector<int> trp(dm.E + 1, 0), tci, tdiag(dm.E, -1), tmap;
  tci.reserve(dm.nnzb);
  tmap.reserve(dm.nnzb);
  for (int e = 0; e < dm.E; ++e) {
    const long long te = tile_of(e);
    for (int kb = rp[e]; kb < rp[e + 1]; ++kb) {
      const int k = ci[kb];
      if (k < 0 || k >= dm.E) return set_err(c, ICX_ERR_INVALID, "block pattern column out of range");
      if (tile_of(k) != te) continue;
      if (k == e) tdiag[e] = (int)tci.size();
      tci.push_back(k);
      tmap.push_back(kb);
    }
    trp[e + 1] = (int)tci.size();
    if (tdiag[e] < 0) return set_err(c, ICX_ERR_INVALID, "block pattern without a diagonal block");
  }
  // levels of the kept lower-triangular dependencies in natural order (on a
  // tile: (i mod s) + (j mod s))
  int nl = 0;
  std::vector<int> lvl(dm.E, 0);
  for (int e = 0; e < dm.E; ++e) {
    for (int kb = trp[e]; kb < tdiag[e]; ++kb) lvl[e] = std::max(lvl[e], lvl[tci[kb]] + 1);
    nl = std::max(nl, lvl[e] + 1);
  }
  IluTilePlan tp;
  tp.lvl_off.assign(nl + 1, 0);
  for (int v : lvl) ++tp.lvl_off[v + 1];
  for (int l = 0; l < nl; ++l) tp.lvl_off[l + 1] += tp.lvl_off[l];
  std::vector<int> order(dm.E), fill(tp.lvl_off.begin(), tp.lvl_off.end() - 1);
  for (int e = 0; e < dm.E; ++e) order[fill[lvl[e]]++] = e;
  tp.nnzb = (int)tci.size();
  // per group: its elements by (level, element), and the level bounds
  std::map<long long, int> gid_of;
  for (int e = 0; e < dm.E; ++e) gid_of.emplace(tile_of(e), 0);
  int ng = 0;
  for (auto& kv : gid_of) kv.second = ng++;
  std::vector<std::array<int, 3>> key(dm.E);
  for (int e = 0; e < dm.E; ++e) key[e] = {gid_of[tile_of(e)], lvl[e], e};
  std::sort(key.begin(), key.end());
  std::vector<int> gtask(8 * (size_t)dm.E), glev, glev_ptr(1, 0);
  for (int p = 0; p < dm.E; ++p) {
    // each sweep row's off-diagonal blocks (kept pattern): forward the ones
    // before the diagonal, backward the ones after it; at most two of each
    // (more: the entry is marked invalid, and the data-flow apply runs instead)
    const int e = key[p][2];
    const int sweeps[2][2] = {{trp[e], tdiag[e]}, {tdiag[e] + 1, trp[e + 1]}};
    for (int sw = 0; sw < 2; ++sw) {
      int* t = &gtask[4 * ((size_t)sw * dm.E + p)];
      const int b0 = sweeps[sw][0], nb = sweeps[sw][1] - b0;
      t[0] = nb > 2 ? -1 : e;
      tp.group_ok = tp.group_ok && nb <= 2;
      t[1] = b0;
      t[2] = nb > 0 ? tci[b0] : -1;
      t[3] = nb > 1 ? tci[b0 + 1] : -1;
    }
    const bool new_group = p == 0 || key[p][0] != key[p - 1][0];
    if (new_group && p > 0) {
      glev.push_back(p);  // the previous group's end
      glev_ptr.push_back((int)glev.size());
    }
    if (new_group || key[p][1] != key[p - 1][1]) glev.push_back(p);
  }
  glev.push_back(dm.E);
  glev_ptr.push_back((int)glev.size());
  tp.ngroups = ng;
  // the same entries by position within the group: {element, k0, k1, 0}
  // (k = -1: no such block); the kept pattern couples only elements of one group
  std::vector<int> gloc(8 * (size_t)dm.E, -1), pos(dm.E), gstart(dm.E);
  for (int p = 0; p < dm.E; ++p) pos[key[p][2]] = p;
  for (int g = 0; g < ng; ++g)
    for (int p = glev[glev_ptr[g]]; p < glev[glev_ptr[g + 1] - 1]; ++p) gstart[p] = glev[glev_ptr[g]];
  for (int sw = 0; sw < 2; ++sw)
    for (int p = 0; p < dm.E; ++p) {
      const int* t = &gtask[4 * ((size_t)sw * dm.E + p)];
      int* l = &gloc[4 * ((size_t)sw * dm.E + p)];
      l[0] = p - gstart[p];
      l[3] = 0;
      for (int j = 0; j < 2; ++j) {
        const int k = t[2 + j];
        l[1 + j] = k < 0 ? -1 : pos[k] - gstart[p];
        if (k >= 0 && gstart[pos[k]] != gstart[p]) tp.group_ok = false;
      }
    }
  for (int g = 0; g < ng; ++g) {
    tp.gmax = std::max(tp.gmax, glev[glev_ptr[g + 1] - 1] - glev[glev_ptr[g]]);
    tp.nlev_max = std::max(tp.nlev_max, glev_ptr[g + 1] - glev_ptr[g] - 1);
  }
  const std::pair<int**, const std::vector<int>*> up[] = {
      {&tp.rowptr, &trp}, {&tp.colidx, &tci}, {&tp.diag, &tdiag}, {&tp.map, &tmap}, {&tp.order, &order},
      {&tp.gtask, &gtask}, {&tp.gloc, &gloc}, {&tp.glev, &glev}, {&tp.glev_ptr, &glev_ptr}};
  for (const auto& u : up) {
    cudaError_t e = cudaMalloc((void**)u.first, sizeof(int) * u.second->size());
    if (e == cudaSuccess) e = cudaMemcpy(*u.first, u.second->data(), sizeof(int) * u.second->size(),
                                         cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      free_tile_plan(tp);
      return set_err(c, ICX_ERR_CUDA, std::string("tiled ILU plan: ") + cudaGetErrorString(e));
    }
  }
  tp.tile = st;
  tp.gen = c->ilu_plan_gen;
  w->tp = std::move(tp);
  return ICX_OK;
}

// the mesh view the block-ILU(0) factors live on: the full pattern, or the
// tiled one when a tile plan is built
icx::DeviceMesh ilu_mesh(const icx_ctx* c) {
  icx::DeviceMesh v = c->dm;
  const IluTilePlan& tp = c->sw->tp;
  if (tp.tile) {
    v.bsr_rowptr = tp.rowptr;
    v.bsr_colidx = tp.colidx;
    v.bsr_diag = tp.diag;
    v.nnzb = tp.nnzb;
  }
  return v;
}

const int* ilu_order(const icx_ctx* c) { return c->sw->tp.tile ? c->sw->tp.order : c->sw->order; }

// NaN when a launch, copy or earlier kernel failed (the CUDA message is kept in c->err)
double dev_norm(icx_ctx* c, const double* x, cudaStream_t s) {
  icx_solver_work* w = c->sw;
  cudaError_t e = icx::la_mdot(w->lw, w->n, x, 0, 1, x, w->dh, s);
  double h = 0.0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, w->dh, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    c->err = std::string("norm: ") + cudaGetErrorString(e);
    return NAN;
  }
  return std::sqrt(h);
}

// FP32 copies of the Jacobian and preconditioner (mixed precision), allocated on first use
icx_status ensure_mixed(icx_ctx* c) {
  icx_solver_work* w = c->sw;
  if (w->vals32) return ICX_OK;
  size_t nv = (size_t)w->nnzb * w->bs * w->bs;
  CK(cudaMalloc((void**)&w->vals32, sizeof(float) * nv));
  CK(cudaMalloc((void**)&w->pc32, sizeof(float) * nv));
  CK(cudaMalloc((void**)&w->uinv32, sizeof(float) * (size_t)c->dm.E * w->bs * w->bs));
  CK(cudaMalloc((void**)&w->V32, sizeof(float) * (size_t)(w->m + 1) * w->n));
  CK(cudaMalloc((void**)&w->vt, sizeof(double) * w->n));
  return ICX_OK;
}

icx_status ensure_bf16(icx_ctx* c) {
  icx_solver_work* w = c->sw;
  if (w->pc16) return ICX_OK;
  size_t nv = (size_t)w->nnzb * w->bs * w->bs;
  CK(cudaMalloc((void**)&w->pc16, sizeof(__nv_bfloat16) * nv));
  CK(cudaMalloc((void**)&w->uinv16, sizeof(__nv_bfloat16) * (size_t)c->dm.E * w->bs * w->bs));
  return ICX_OK;
}

cudaError_t diag_apply(icx_ctx* c, bool mixed, const double* D, const float* D32, const double* x, double* z,
                       cudaStream_t s) {
  return mixed ? icx::la_block_diag_apply_f32(c->dm.E, c->sw->bs, D32, x, z, s)
               : icx::la_block_diag_apply(c->dm.E, c->sw->bs, D, x, z, s);
}

cudaError_t tri_rows(icx_ctx* c, bool mixed, bool lower, const double* v, const double* x0, double* y,
                     cudaStream_t s) {
  icx_solver_work* w = c->sw;
  const icx::DeviceMesh dm = ilu_mesh(c);
  return mixed ? icx::la_tri_rows_f32(dm, lower, w->pc32, v, x0, -1.0, y, s)
               : icx::la_tri_rows(dm, lower, w->pc, v, x0, -1.0, y, s);
}

// the data-flow block-ILU(0) apply with the context's launch shape. Each
// apply adds an element's task count to its counters and waits for
// epoch x task count, so a change of rows per task (FP64 and FP32 applies may
// differ) first zeroes the counters, in stream order
cudaError_t ilu_flow(icx_ctx* c, bool mixed, const double* x, double* z, cudaStream_t s) {
  icx_solver_work* w = c->sw;
  const icx::DeviceMesh dm = ilu_mesh(c);
  const int* order = ilu_order(c);
  const int pi = mixed ? 1 : 0;
  const int rows = dm.tile.flow_rows[pi] ? dm.tile.flow_rows[pi] : icx::flow_rows_default(w->bs);
  const int gsched = icx::ilu_schedule(dm.tile, pi, true);
  if (w->tp.tile && w->tp.group_ok && gsched >= 3) {
    // tiled / grouped factors: one CTA per group, no waits across CTAs
    const IluTilePlan& tp = w->tp;
    const icx::IluGroupShape gs{tp.ngroups, tp.gmax, tp.nlev_max, gsched, tp.gloc};
    const int ctas = dm.tile.flow_ctas[pi];
    // BF16 factors: the one-lane-per-row form where it fits, else the FP32
    // copies. Its CTA size follows the group size (measured at 256 x 256,
    // p = 2: 8 x 8 tiles 0.159 ms with 128 threads against 0.191 with 256;
    // 16 x 16 tiles 0.240 ms with 256 against 0.322 with 128)
    if (mixed && w->bf16 && w->pc16 && icx::group_rows_bf16_fits(dm, gs)) {
      const int ctas16 = tp.gmax <= 64 ? 3 : tp.gmax <= 256 ? 2 : 1;
      return icx::la_ilu_apply_groups_bf16(dm, gs, tp.gtask, tp.glev, tp.glev_ptr, ctas16, w->pc16, w->uinv16, x,
                                           z, w->pct, w->pc_err, s);
    }
    return mixed ? icx::la_ilu_apply_groups_f32(dm, gs, tp.gtask, tp.glev, tp.glev_ptr, rows, ctas, w->pc32,
                                                w->uinv32, x, z, w->pct, w->pc_err, s)
                 : icx::la_ilu_apply_groups(dm, gs, tp.gtask, tp.glev, tp.glev_ptr, rows, ctas, w->pc, w->uinv,
                                            x, z, w->pct, w->pc_err, s);
  }
  // the sentinel schedule uses neither the counters nor the epoch
  const bool sen = icx::flow_sentinel(dm.tile, pi);
  if (!sen && rows != w->flow_rows) {
    cudaError_t e = cudaMemsetAsync(w->cnt, 0, sizeof(unsigned) * 2 * dm.E, s);
    if (e != cudaSuccess) return e;
    w->epoch = 0;
    w->flow_rows = rows;
  }
  const unsigned epoch = sen ? w->epoch : ++w->epoch;
  if (mixed)
    return icx::la_ilu_apply_flow_f32(dm, order, w->pc32, w->uinv32, x, z, w->pct, w->cnt, w->cnt + dm.E,
                                      epoch, w->pc_err, s);
  return icx::la_ilu_apply_flow(dm, order, w->pc, w->uinv, x, z, w->pct, w->cnt, w->cnt + dm.E, epoch,
                                w->pc_err, s);
}

// z = M^-1 x (mixed: from the FP32 copies, FP32 accumulation)
cudaError_t apply_pc(icx_ctx* c, int kind, bool mixed, const double* x, double* z, cudaStream_t s) {
  icx_solver_work* w = c->sw;
  const icx::DeviceMesh& dm = c->dm;
  if (kind == 1) return diag_apply(c, mixed, w->pc, w->pc32, x, z, s);
  if (kind == 3) {
    // one Richardson step on block-Jacobi: z = G (2x - J G x)
    cudaError_t e = diag_apply(c, mixed, w->pc, w->pc32, x, w->pct, s);
    if (e == cudaSuccess)
      e = mixed ? icx::launch_bsr_spmv_f32(dm, w->vals32, w->pct, w->pct2, s)
                : icx::launch_bsr_spmv(dm, w->vals, w->pct, w->pct2, s);
    if (e == cudaSuccess) e = icx::la_axpby(w->n, 2.0, x, -1.0, w->pct2, s);
    if (e == cudaSuccess) e = diag_apply(c, mixed, w->pc, w->pc32, w->pct2, z, s);
    return e;
  }
  if (kind == 5) {
    // learned: z = (I + C) y, y from the ILU(0) factors by `sweeps` Jacobi
    // sweeps per triangle, or by the exact triangular solves when sweeps = 0;
    // a model whose output layer is zero (C = 0) is its base
    if (icx::lpc_zero_correction(c)) return apply_pc(c, w->sweeps > 0 ? 4 : 2, mixed, x, z, s);
    cudaError_t e = apply_pc(c, w->sweeps > 0 ? 4 : 2, mixed, x, w->pct4, s);
    if (e == cudaSuccess) e = icx::lpc_apply(c, w->pct4, z, s);
    return e;
  }
  if (kind == 4) {
    // ILU(0) factors, each triangular solve replaced by `sweeps` Jacobi sweeps:
    // f <- x - L f, then y <- inv(U_ee) f - (inv(U_ee) U) y
    const int sw = w->sweeps;
    const double* cur = x;
    cudaError_t e = cudaSuccess;
    for (int k = 1; k <= sw && e == cudaSuccess; ++k) {
      double* out = (k & 1) ? w->pct : w->pct2;
      e = tri_rows(c, mixed, true, cur, x, out, s);
      cur = out;
    }
    if (e == cudaSuccess) e = diag_apply(c, mixed, w->uinv, w->uinv32, cur, sw == 0 ? z : w->pct3, s);
    cur = w->pct3;
    for (int k = 1; k <= sw && e == cudaSuccess; ++k) {
      double* out = k == sw ? z : ((k & 1) ? w->pct : w->pct2);
      e = tri_rows(c, mixed, false, cur, w->pct3, out, s);
      cur = out;
    }
    return e;
  }
  if (kind == 2) {
    if (w->rows_ok && w->schedule == 2 && !w->tp.tile) {
      const unsigned ep = w->epoch_rows + 1;
      cudaError_t e = mixed ? icx::la_ilu_apply_rows_f32(dm, c->nx, c->ny, w->pc32, w->uinv32, x, z, w->pct,
                                                         w->cnt_rows, w->cnt_rows + dm.E, ep, w->pc_err, s)
                            : icx::la_ilu_apply_rows(dm, c->nx, c->ny, w->pc, w->uinv, x, z, w->pct, w->cnt_rows,
                                                     w->cnt_rows + dm.E, ep, w->pc_err, s);
      if (e == cudaSuccess) w->epoch_rows = ep;
      if (e != cudaErrorNotSupported) return e;
      w->rows_ok = false;  // the rows cannot all be resident: data-flow apply from now on
    }
    return ilu_flow(c, mixed, x, z, s);
  }
  return cudaMemcpyAsync(z, x, sizeof(double) * w->n, cudaMemcpyDeviceToDevice, s);
}

// builds the preconditioner from w->vals (in FP64; mixed: then rounded to FP32,
// together with the Jacobian itself)
cudaError_t build_pc_impl(icx_ctx* c, int kind, bool mixed, cudaStream_t s) {
  icx_solver_work* w = c->sw;
  const icx::DeviceMesh& dm = c->dm;
  const long long nv = (long long)dm.nnzb * w->bs * w->bs, nd = (long long)dm.E * w->bs * w->bs;
  cudaError_t e = cudaMemsetAsync(w->flag, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  const bool jac = kind == 1 || kind == 3, ilu = kind == 2 || kind == 4 || kind == 5;
  if (kind == 5 && !icx::lpc_zero_correction(c) && (e = icx::lpc_build(c, w->vals, s)) != cudaSuccess) return e;
  if (jac) e = icx::la_block_invert(dm.E, w->bs, w->vals, dm.bsr_diag, w->pc, w->flag, s);
  long long nv_pc = nv;
  if (ilu) {
    if (w->tp.tile) {
      // the kept blocks, compacted into the tiled pattern's order
      const icx::DeviceMesh dt = ilu_mesh(c);
      nv_pc = (long long)dt.nnzb * w->bs * w->bs;
      e = icx::la_gather_blocks(dt.nnzb, w->bs, w->vals, w->tp.map, w->pc, s);
      if (e == cudaSuccess) e = icx::la_ilu_factor(dt, w->tp.order, w->tp.lvl_off, w->pc, w->uinv, w->flag, s);
    } else {
      e = cudaMemcpyAsync(w->pc, w->vals, sizeof(double) * nv, cudaMemcpyDeviceToDevice, s);
      if (e == cudaSuccess) e = icx::la_ilu_factor(dm, w->order, w->lvl_off, w->pc, w->uinv, w->flag, s);
    }
  }
  if (e != cudaSuccess || !mixed) return e;
  e = icx::la_d2f(nv, w->vals, w->vals32, s);
  if (e == cudaSuccess && jac) e = icx::la_d2f(nd, w->pc, w->pc32, s);
  if (e == cudaSuccess && ilu) e = icx::la_d2f(nv_pc, w->pc, w->pc32, s);
  if (e == cudaSuccess && ilu) e = icx::la_d2f(nd, w->uinv, w->uinv32, s);
  if (e == cudaSuccess && ilu && w->bf16 && w->pc16) {
    e = icx::la_d2bf(nv_pc, w->pc, w->pc16, s);
    if (e == cudaSuccess) e = icx::la_d2bf(nd, w->uinv, w->uinv16, s);
  }
  return e;
}

// the preconditioner for the context's current ILU tiling (the tiled plan is
// built on the first use of a new tile size)
cudaError_t build_pc(icx_ctx* c, int kind, bool mixed, cudaStream_t s) {
  if (kind == 2 || kind == 4 || kind == 5) {
    if (ensure_ilu_plan(c) != ICX_OK) return cudaErrorInvalidValue;  // c->err says why
  }
  return build_pc_impl(c, kind, mixed, s);
}

// x = J^-1 b by GMRES(m) on the BSR Jacobian, right preconditioning
// (mixed: operator and preconditioner from the FP32 copies; the Krylov
// vectors, Hessenberg and Givens rotations stay FP64)
icx_status gmres(icx_ctx* c, int pc, bool mixed, int m, int maxit, double rtol, const double* b, double* x,
                 int* iters, double* relres, cudaStream_t s, double* samples = nullptr, int sample_cap = 0,
                 int sample_every = 0, int* sample_count = nullptr) {
  icx_solver_work* w = c->sw;
  const icx::DeviceMesh& dm = c->dm;
  icx::KrylovBuffers kb;
  kb.n = w->n;
  kb.m = m;
  kb.V = w->V;
  kb.w = w->w;
  kb.z = w->z;
  kb.r = w->r;
  kb.dh = w->dh;
  kb.lw = &w->lw;
  kb.samples = samples;
  kb.sample_cap = sample_cap;
  kb.sample_every = sample_every;
  if (mixed && w->V32 && m <= w->m) {
    // the Krylov basis in FP32 (inner products and updates in FP64)
    kb.V32 = w->V32;
    kb.vt = w->vt;
  }
  // the parallel and learned preconditioners give up on a stalled solve
  // (block-ILU(0) then takes the step): under 10 % residual reduction over
  // 20 restart cycles
  kb.stall_cycles = pc >= 3 ? 20 : 0;
  kb.cgs_passes = w->cgs_passes;
  struct CountOut {
    int* dst;
    icx::KrylovBuffers* kb;
    ~CountOut() { if (dst) *dst = kb->sample_count; }
  } count_out{sample_count, &kb};
  icx::LinOp A = [&](const double* xin, double* yout, cudaStream_t st) -> cudaError_t {
    if (w->fd_on) {
      // (R(u + h v) - R(u)) / h, h from |v| on the device; the perturbed
      // state and residual in ustep / rwork (free while the solve runs)
      cudaError_t e = icx::la_mdot(w->lw, w->n, xin, 0, 1, xin, w->fd_slot, st);
      if (e == cudaSuccess) e = icx::la_fd_perturb(w->n, w->fd_u, xin, w->fd_slot, w->ustep, st);
      if (e == cudaSuccess) e = icx::launch_residual(dm, c->phys, w->ustep, w->rwork, st);
      if (e == cudaSuccess) e = icx::la_fd_diff(w->n, w->rwork, w->fd_r, w->fd_slot, yout, st);
      return e;
    }
    return mixed ? icx::launch_bsr_spmv_f32(dm, w->vals32, xin, yout, st) : icx::launch_bsr_spmv(dm, w->vals, xin, yout, st);
  };
  icx::LinOp M = [&](const double* xin, double* yout, cudaStream_t st) { return apply_pc(c, pc, mixed, xin, yout, st); };
  // CUDA graphs of the Arnoldi steps where the preconditioner apply launches
  // the same kernels with the same arguments every time: none, block-Jacobi,
  // the two-step and sweep forms, and block-ILU(0) on the sentinel schedule
  // (the counter schedule passes a new epoch to every apply, the row schedule
  // likewise; the learned preconditioner is left out)
  const bool graphable = icx::solver_graphable(c, pc, mixed);
  if (graphable) {
    const icx::TileChoice& t = dm.tile;
    const int pi = mixed ? 1 : 0;
    unsigned long long key = 1469598103934665603ull;  // FNV-1a over what the step's launches depend on
    for (long long v : {(long long)pc, (long long)mixed, (long long)w->sweeps, (long long)m, (long long)t.flow_rows[pi],
                        (long long)t.flow_ctas[pi], (long long)t.flow_sched[pi], (long long)(uintptr_t)dm.bsr_rowptr,
                        (long long)(uintptr_t)dm.bsr_colidx, (long long)(uintptr_t)dm.bsr_diag,
                        (long long)(uintptr_t)w->order, (long long)w->tp.tile, (long long)(uintptr_t)w->tp.order,
                        (long long)w->fd_on, (long long)(uintptr_t)w->fd_u, (long long)(uintptr_t)w->fd_r,
                        (long long)w->bf16, (long long)w->cgs_passes})
      key = (key ^ (unsigned long long)v) * 1099511628211ull;
    kb.graphs = &w->graphs;
    kb.graph_key = key | 1;
  }
  icx_status st = icx::gmres_op(kb, A, pc ? &M : nullptr, maxit, rtol, b, x, iters, relres, s, &c->err);
  w->graph_steps += kb.graph_launches;
  if (st != ICX_OK) {
    // a non-finite value may come from a failed kernel: report that first
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string("linear solve: ") + cudaGetErrorString(e));
    return st;  // c->err holds the failing call
  }
  int perr = 0;
  CK(cudaMemcpyAsync(&perr, w->pc_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (perr) {
    // the counters are inconsistent after an abandoned apply: start over
    cudaMemsetAsync(w->pc_err, 0, sizeof(int), s);
    cudaMemsetAsync(w->cnt, 0, sizeof(unsigned) * 2 * dm.E, s);
    cudaMemsetAsync(w->cnt_rows, 0, sizeof(unsigned) * 2 * dm.E, s);
    w->epoch = 0;
    w->epoch_rows = 0;
    return set_err(c, ICX_ERR_CUDA, perr == 2 ? "block-ILU apply: block index out of range"
                                              : "block-ILU apply: a dependency wait timed out");
  }
  return st;
}

// wolfe_ls / zoom / corrigan_ls of the reference (nonlinear_solver_utils.hpp:83-191)
double finite_difference(const std::function<double(double)>& f, double eps, double x) {
  double a = f(x), b = f(x + eps);
  return (b - a) / eps;
}

double zoom(const std::function<double(double)>& f, double lo, double hi, int kmax, double c1, double c2) {
  const double EPS = std::sqrt(DBL_EPSILON);
  for (int k = 0; k < kmax; ++k) {
    double phi_lo = f(lo), dphi_lo = finite_difference(f, EPS, lo);
    double phi_hi = f(hi), dphi_hi = finite_difference(f, EPS, hi);
    double d1 = dphi_lo + dphi_hi - 3 * (phi_lo - phi_hi) / (lo - hi);
    double d2 = std::sqrt(std::max(d1 * d1 - dphi_lo * dphi_hi, 1e-8));
    d2 = std::copysign(d2, hi - lo);
    double aj = hi - (hi - lo) * ((dphi_hi + d2 - d1) / (dphi_hi - dphi_lo + 2 * d2));
    double phi_aj = f(aj);
    double dphi_0 = finite_difference(f, EPS, 0.0);
    if (phi_aj > (f(0) + c1 * aj * dphi_0) || phi_aj >= phi_lo) {
      hi = aj;
    } else {
      double dphi_aj = finite_difference(f, EPS, aj);
      if (std::fabs(dphi_aj) <= -c2 * dphi_0) return aj;
      if (dphi_aj * (hi - lo) >= 0) hi = lo;
      lo = aj;
    }
  }
  return 0.5 * (lo + hi);
}

double wolfe_ls(const std::function<double(double)>& f, double alpha_max, double alpha1, int kmax, double c1,
                double c2) {
  const double EPS = std::sqrt(DBL_EPSILON);
  double a_im1 = 0, a_i = alpha1;
  double phi_0 = f(0);
  double dphi_0 = finite_difference(f, EPS, 0.0);
  for (int k = 0; k < kmax; ++k) {
    double phi_i = f(a_i), phi_im1 = f(a_im1);
    if (phi_i > phi_0 + c1 * a_i * dphi_0 || (phi_i >= phi_im1 && k > 0)) return zoom(f, a_im1, a_i, kmax, c1, c2);
    double dphi_i = finite_difference(f, EPS, a_i);
    if (std::fabs(dphi_i) <= -c2 * dphi_0) return a_i;
    if (dphi_i >= 0) return zoom(f, a_i, a_im1, kmax, c1, c2);
    double t = 0.5 * (a_i + alpha_max);
    a_im1 = a_i;
    a_i = t;
  }
  return a_i;
}

double corrigan_ls(const std::function<double(double)>& f, double alpha_max, double alpha1, int kmax,
                   double alpha_min) {
  double alpha_a = alpha_min, alpha_b = alpha_max, alpha = alpha1;
  for (int k = 0; k < kmax; ++k) {
    double phi_0 = f(0);
    if (k > 0) alpha = (alpha_a + alpha_b) / 2;
    double phi_star = f(alpha);
    if (std::fabs(phi_star) < std::fabs(phi_0)) {
      if (alpha == alpha1) break;
      alpha_a = alpha;
    } else {
      alpha_b = alpha;
    }
  }
  return alpha;
}

}  // namespace

namespace icx {
void free_solver_work(icx_ctx* c) {
  if (!c || !c->sw) return;
  icx_solver_work* w = c->sw;
  void* ptrs[] = {w->pc16, w->uinv16, w->V32, w->vt, w->vals32, w->pc32, w->uinv32, w->vals, w->pc, w->uinv, w->V, w->w, w->z, w->r, w->res, w->du,
                  w->ustep, w->rwork, w->pct, w->pct2, w->pct3, w->pct4, w->order, w->cnt, w->cnt_rows, w->pc_err,
                  w->dh, w->flag, w->lw.partial};
  w->graphs.release();
  for (void* p : ptrs)
    if (p) cudaFree(p);
  free_tile_plan(w->tp);
  delete w;
  c->sw = nullptr;
}
}  // namespace icx

extern "C" {

icx_status icx_form_jacobian_fd(icx_ctx* c, const double* d_u, double* d_res, double* d_vals, double eps,
                                void* stream) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !d_res || !d_vals) return set_err(c, ICX_ERR_INVALID, "null device pointer");
  if (!(eps > 0.0)) eps = std::sqrt(DBL_EPSILON);
  cudaError_t e = icx::launch_jacobian_fd(c->dm, c->phys, d_u, d_res, d_vals, eps, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string("jacobian kernels: ") + cudaGetErrorString(e));
  return ICX_OK;
}

icx_status icx_form_jacobian_fd_f32(icx_ctx* c, const double* d_u, double* d_res, float* d_vals32, void* stream) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !d_res || !d_vals32) return set_err(c, ICX_ERR_INVALID, "null device pointer");
  cudaError_t e = icx::launch_jacobian_fd_f32(c->dm, c->phys, d_u, d_res, d_vals32, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string("jacobian kernels: ") + cudaGetErrorString(e));
  return ICX_OK;
}

icx_status icx_bsr_spmv(icx_ctx* c, const double* d_vals, const double* d_x, double* d_y, void* stream) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_vals || !d_x || !d_y) return set_err(c, ICX_ERR_INVALID, "null device pointer");
  cudaError_t e = icx::launch_bsr_spmv(c->dm, d_vals, d_x, d_y, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string("spmv: ") + cudaGetErrorString(e));
  return ICX_OK;
}

icx_status icx_newton_default_options(icx_newton_options* o) {
  if (!o) return ICX_ERR_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->tau_abs = 1e-10;
  o->tau_rel = 0.0;
  o->kmax = 20;
  o->linesearch = 1;         // wolfe_linesearch defaults (nonlinear_solver_utils.hpp:207-233)
  o->ls_max_it = 20;
  o->ls_alpha_initial = 1.0;
  o->ls_alpha_max = 10.0;
  o->ls_alpha_min = 0.0;
  o->ls_c1 = 1e-4;
  o->ls_c2 = 0.9;
  o->gmres_restart = 30;     // PETSc KSPGMRES default restart
  o->gmres_max_it = 2000;
  o->gmres_rtol = 1e-5;      // PETSc KSP default relative tolerance
  o->preconditioner = 2;     // block-ILU(0)
  o->verbosity = 0;
  o->precision = 0;          // all FP64
  o->pc_sweeps = 2;
  o->cuda_graphs = 1;
  o->ilu_tile = 0;           // block-ILU(0) over the whole grid in natural order
  o->matrix_free = 0;        // the assembled Jacobian's BSR product
  o->gmres_cgs_refine = 1;   // classical Gram-Schmidt with a second pass every step
  return ICX_OK;
}

icx_status icx_set_ilu_tile(icx_ctx* c, int tile) {
  if (!c) return ICX_ERR_INVALID;
  if (tile < 0 || tile > (1 << 20)) return set_err(c, ICX_ERR_INVALID, "ILU tile side must be in 0..2^20");
  if (tile != c->ilu_tile) ++c->ilu_plan_gen;
  c->ilu_tile = tile;
  return ICX_OK;
}

icx_status icx_set_ilu_groups(icx_ctx* c, const int* groups) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (groups) c->ilu_groups.assign(groups, groups + c->dm.E);
  else c->ilu_groups.clear();
  ++c->ilu_plan_gen;
  return ICX_OK;
}

icx_status icx_pc_factor(icx_ctx* c, const double* d_vals, int precision) {
  if (!c || !c->ready || !d_vals) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed / null pointer");
  if (precision < 0 || precision > 1) return set_err(c, ICX_ERR_INVALID, "precision 0 or 1");
  icx_status st = ensure_work(c, 30);
  if (st != ICX_OK) return st;
  const bool mixed = precision == 1;
  if (mixed && (st = ensure_mixed(c)) != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  cudaStream_t s = 0;
  CK(cudaMemcpyAsync(w->vals, d_vals, sizeof(double) * (size_t)c->dm.nnzb * w->bs * w->bs, cudaMemcpyDeviceToDevice,
                     s));
  CK(build_pc(c, 2, mixed, s));
  int fl = 0;
  CK(cudaMemcpyAsync(&fl, w->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  SYNC_AT("preconditioner");
  if (fl == 2) return set_err(c, ICX_ERR_CUDA, "block-ILU factorization: block index out of range");
  if (fl == 1) return set_err(c, ICX_ERR_NONFINITE, "block-ILU factorization: singular diagonal block");
  return ICX_OK;
}

icx_status icx_pc_apply(icx_ctx* c, const double* d_x, double* d_y, int precision, void* stream) {
  if (!c || !c->sw || !d_x || !d_y || d_x == d_y) return set_err(c, ICX_ERR_INVALID, "no factors / bad pointers");
  if (precision == 1 && !c->sw->vals32) return set_err(c, ICX_ERR_INVALID, "no FP32 factors (icx_pc_factor)");
  CK(apply_pc(c, 2, precision == 1, d_x, d_y, (cudaStream_t)stream));
  return ICX_OK;
}

int icx_get_ilu_tile(const icx_ctx* c) { return c ? c->ilu_tile : -1; }

icx_status icx_gmres_solve(icx_ctx* c, const double* d_vals, const double* d_b, double* d_x, int restart, int maxit,
                           double rtol, int preconditioner, int* iterations, double* relres, void* stream) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_vals || !d_b || !d_x) return set_err(c, ICX_ERR_INVALID, "null device pointer");
  if (restart < 1 || restart > 60 || preconditioner < 0 || preconditioner > 4)
    return set_err(c, ICX_ERR_INVALID, "restart must be in 1..60 and preconditioner in 0..4");
  cudaStream_t s = (cudaStream_t)stream;
  icx_status st = ensure_work(c, restart);
  if (st != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  CK(cudaMemcpyAsync(w->vals, d_vals, sizeof(double) * (size_t)c->dm.nnzb * w->bs * w->bs, cudaMemcpyDeviceToDevice,
                     s));
  CK(build_pc(c, preconditioner, false, s));
  int it = 0;
  double rr = 0.0;
  st = gmres(c, preconditioner, false, restart, maxit, rtol, d_b, d_x, &it, &rr, s);
  if (iterations) *iterations = it;
  if (relres) *relres = rr;
  if (st != ICX_OK) return st;
  return rr <= rtol ? ICX_OK : ICX_ERR_NOT_CONVERGED;
}

icx_status icx_ilu_apply(icx_ctx* c, const double* d_vals, const double* d_x, double* d_y, int precision,
                         int schedule, int repeat, double* ms_per_apply) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_vals || !d_x || !d_y || d_x == d_y) return set_err(c, ICX_ERR_INVALID, "null or aliased device pointer");
  if (precision < 0 || precision > 2 || schedule < 0 || schedule > 2 || repeat < 1)
    return set_err(c, ICX_ERR_INVALID, "precision 0..2, schedule 0..2, repeat >= 1");
  cudaStream_t s = 0;
  icx_status st = ensure_work(c, 30);
  if (st != ICX_OK) return st;
  const bool mixed = precision >= 1;
  if (mixed && (st = ensure_mixed(c)) != ICX_OK) return st;
  if (precision == 2 && (st = ensure_bf16(c)) != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  struct Bf16Scope {
    icx_solver_work* w;
    ~Bf16Scope() { w->bf16 = false; }
  } bf16_scope{w};
  w->bf16 = precision == 2;
  if (schedule == 2 && !w->rows_ok)
    return set_err(c, ICX_ERR_UNSUPPORTED, "row-pipelined apply needs one structured grid with the 5-point pattern");
  CK(cudaMemcpyAsync(w->vals, d_vals, sizeof(double) * (size_t)c->dm.nnzb * w->bs * w->bs, cudaMemcpyDeviceToDevice,
                     s));
  CK(build_pc(c, 2, mixed, s));
  w->schedule = schedule;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (ms_per_apply) {
    CK(cudaEventCreate(&ev[0]));
    CK(cudaEventCreate(&ev[1]));
    CK(cudaEventRecord(ev[0], s));
  }
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < repeat && e == cudaSuccess; ++k) e = apply_pc(c, 2, mixed, d_x, d_y, s);
  w->schedule = 0;
  if (ms_per_apply && e == cudaSuccess) {
    float ms = 0.f;
    e = cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
    *ms_per_apply = (double)ms / repeat;
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  CK(e);
  int perr = 0;
  CK(cudaMemcpyAsync(&perr, w->pc_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (perr) {
    cudaMemsetAsync(w->pc_err, 0, sizeof(int), s);
    cudaMemsetAsync(w->cnt, 0, sizeof(unsigned) * 2 * c->dm.E, s);
    cudaMemsetAsync(w->cnt_rows, 0, sizeof(unsigned) * 2 * c->dm.E, s);
    w->epoch = 0;
    w->epoch_rows = 0;
    return set_err(c, ICX_ERR_CUDA, perr == 2 ? "block-ILU apply: block index out of range"
                                              : "block-ILU apply: a dependency wait timed out");
  }
  return ICX_OK;
}

icx_status icx_krylov_samples(icx_ctx* c, const double* d_vals, const double* d_b, double* d_x, int restart, int maxit,
                              double rtol, int preconditioner, int every, int capacity, double* d_samples,
                              int* n_samples, int* iterations, double* relres) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_vals || !d_b || !d_x || !d_samples || capacity < 1 || every < 1)
    return set_err(c, ICX_ERR_INVALID, "null pointer, capacity < 1 or every < 1");
  if (restart < 1 || restart > 60 || preconditioner < 0 || preconditioner > 4)
    return set_err(c, ICX_ERR_INVALID, "restart must be in 1..60 and preconditioner in 0..4");
  cudaStream_t s = 0;
  icx_status st = ensure_work(c, restart);
  if (st != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  CK(cudaMemcpyAsync(w->vals, d_vals, sizeof(double) * (size_t)c->dm.nnzb * w->bs * w->bs, cudaMemcpyDeviceToDevice,
                     s));
  CK(build_pc(c, preconditioner, false, s));
  int it = 0, cnt = 0;
  double rr = 0.0;
  st = gmres(c, preconditioner, false, restart, maxit, rtol, d_b, d_x, &it, &rr, s, d_samples, capacity, every, &cnt);
  SYNC_AT("krylov samples");
  if (n_samples) *n_samples = cnt;
  if (iterations) *iterations = it;
  if (relres) *relres = rr;
  return st;
}

icx_status icx_newton_solve(icx_ctx* c, double* d_u, const icx_newton_options* opt, icx_newton_report* rep) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !opt) return set_err(c, ICX_ERR_INVALID, "null argument");
  if (opt->gmres_restart < 1 || opt->gmres_restart > 60) return set_err(c, ICX_ERR_INVALID, "restart in 1..60");
  cudaStream_t s = 0;
  if (opt->precision < 0 || opt->precision > 3) return set_err(c, ICX_ERR_INVALID, "precision must be 0 to 3");
  if (opt->preconditioner < 0 || opt->preconditioner > 5) return set_err(c, ICX_ERR_INVALID, "preconditioner in 0..5");
  if (opt->preconditioner >= 4 && (opt->pc_sweeps < 0 || opt->pc_sweeps > 16))
    return set_err(c, ICX_ERR_INVALID, "pc_sweeps in 0..16");
  if (opt->preconditioner == 5 && !c->lpc)
    return set_err(c, ICX_ERR_INVALID, "preconditioner 5 needs a learned model (icx_lpc_attach)");
  if (opt->ilu_tile > (1 << 20)) return set_err(c, ICX_ERR_INVALID, "ILU tile side must be at most 2^20");
  if (opt->ilu_tile >= 0) c->ilu_tile = opt->ilu_tile;  // negative: keep the context's tiling
  icx_status st = ensure_work(c, opt->gmres_restart);
  if (st != ICX_OK) return st;
  c->sw->sweeps = opt->pc_sweeps;
  c->sw->graphs_on = opt->cuda_graphs != 0;
  const long long graph_steps0 = c->sw->graph_steps;
  const bool mixed = opt->precision >= 1;
  const bool quad32 = opt->precision == 2;
  if (mixed && (st = ensure_mixed(c)) != ICX_OK) return st;
  if (opt->precision == 3 && (st = ensure_bf16(c)) != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  // precision 3: BF16 copies of the ILU factors for this solve
  struct Bf16Scope {
    icx_solver_work* w;
    ~Bf16Scope() {
      w->bf16 = false;
      w->cgs_passes = 2;
    }
  } bf16_scope{w};
  w->bf16 = opt->precision == 3;
  w->cgs_passes = opt->gmres_cgs_refine ? 2 : 1;
  // a learned model whose output layer is zero is its base preconditioner,
  // so the solve is the base's: block-ILU(0) (sweeps = 0) or its Jacobi-sweep
  // form, without the stall test and fallback kept for a correction that
  // may not converge
  const int pc_kind = opt->preconditioner == 5 && icx::lpc_zero_correction(c) ? (opt->pc_sweeps > 0 ? 4 : 2)
                                                                             : opt->preconditioner;
  long long n = w->n;
  icx_newton_report local{};
  icx_newton_report* R = rep ? rep : &local;
  std::memset(R, 0, sizeof(*R));
  const double eps = std::sqrt(DBL_EPSILON);
  const size_t nvals = (size_t)w->nnzb * w->bs * w->bs;
  // FP64 residual and the Jacobian (FP32 quadrature: formed in FP32, widened
  // for the FP64 factorisation)
  auto linearise = [&]() -> cudaError_t {
    if (!quad32) return icx::launch_jacobian_fd(c->dm, c->phys, d_u, w->res, w->vals, eps, s);
    cudaError_t e = icx::launch_jacobian_fd_f32(c->dm, c->phys, d_u, w->res, w->vals32, s);
    return e == cudaSuccess ? icx::la_f2d((long long)nvals, w->vals32, w->vals, s) : e;
  };
  // residual and Jacobian at the initial state (petsc_newton.hpp:211-221)
  CK(linearise());
  double r0 = dev_norm(c, w->res, s);
  R->r0 = r0;
  R->residual_history[0] = r0;
  if (!std::isfinite(r0)) {
    SYNC_AT("initial residual");
    return set_err(c, ICX_ERR_NONFINITE, "non-finite initial residual");
  }
  double tau = opt->tau_abs + opt->tau_rel * r0;
  double rk = r0;
  int k = 0;
  bool converged = rk <= tau;
  for (; k < opt->kmax && !converged; ++k) {
    CK(build_pc(c, pc_kind, mixed, s));
    {
      int fl = 0;
      CK(cudaMemcpyAsync(&fl, w->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
      SYNC_AT("preconditioner");
      if (fl == 2) return set_err(c, ICX_ERR_CUDA, "block-ILU factorization: block index out of range");
    }
    // the matrix-free operator at this state: c = sqrt(eps) (sqrt(n) + |u|)
    struct FdScope {
      icx_solver_work* w;
      ~FdScope() { w->fd_on = false; }
    } fd_scope{w};
    if (opt->matrix_free) {
      const double cval = eps * (std::sqrt((double)n) + dev_norm(c, d_u, s));
      w->fd_slot = w->dh + 3 * (w->m + 2);
      CK(cudaMemcpyAsync(w->fd_slot + 1, &cval, sizeof(double), cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
      w->fd_u = d_u;
      w->fd_r = w->res;
      w->fd_on = true;
    }
    int it = 0;
    double rr = 0.0;
    st = gmres(c, pc_kind, mixed, opt->gmres_restart, opt->gmres_max_it, opt->gmres_rtol, w->res, w->du,
               &it, &rr, s);
    if (st != ICX_OK) return st;
    R->linear_iterations_total += it;
    if (k < 64) R->linear_iterations[k] = it;
    if (pc_kind >= 3 && !(rr <= opt->gmres_rtol)) {
      // the parallel / learned preconditioner missed the linear tolerance:
      // this step is solved again with block-ILU(0)
      ++R->pc_fallbacks;
      CK(build_pc(c, 2, mixed, s));
      st = gmres(c, 2, mixed, opt->gmres_restart, opt->gmres_max_it, opt->gmres_rtol, w->res, w->du, &it, &rr, s);
      if (st != ICX_OK) return st;
      R->linear_iterations_total += it;
      if (k < 64) R->linear_iterations[k] += it;
    }
    double alpha = 1.0;
    if (opt->linesearch != 0) {
      // phi(alpha) = |R(u - alpha du)|_2, non-finite -> 1e9 (petsc_newton.hpp:262-293)
      std::function<double(double)> phi = [&](double a) -> double {
        icx::la_xpay(n, d_u, -a, w->du, w->ustep, s);
        icx::launch_residual(c->dm, c->phys, w->ustep, w->rwork, s);
        double v = dev_norm(c, w->rwork, s);
        return std::isfinite(v) ? v : 1e9;
      };
      if (opt->linesearch == 1)
        alpha = wolfe_ls(phi, opt->ls_alpha_max, opt->ls_alpha_initial, opt->ls_max_it, opt->ls_c1, opt->ls_c2);
      else
        alpha = corrigan_ls(phi, opt->ls_alpha_max, opt->ls_alpha_initial, opt->ls_max_it, opt->ls_alpha_min);
    }
    SYNC_AT("line search");
    CK(icx::la_axpby(n, -alpha, w->du, 1.0, d_u, s));
    CK(linearise());
    rk = dev_norm(c, w->res, s);
    if (k + 1 < 64) {
      R->residual_history[k + 1] = rk;
      R->alpha_history[k] = alpha;
    }
    if (opt->verbosity > 0) std::printf("newton %d: |r| = %.6e alpha = %.4f gmres its = %d\n", k, rk, alpha, it);
    if (!std::isfinite(rk)) {
      SYNC_AT("residual");
      return set_err(c, ICX_ERR_NONFINITE, "non-finite residual");
    }
    converged = rk <= tau;
  }
  CK(cudaStreamSynchronize(s));
  R->iterations = k;
  R->converged = converged;
  R->r_final = rk;
  R->graph_steps = (int)(c->sw->graph_steps - graph_steps0);
  return converged ? ICX_OK : ICX_ERR_NOT_CONVERGED;
}
}

// ---------------------------------------------------------------------------
// Matrix-free Newton-Krylov (MFNK, src/solvers/include/iceicle/
// matrix_free_newton_krylov.hpp:62-365) on the PDE unknowns: each Krylov
// product is the one-sided difference J p ~ (R(u + eps p) - R(u)) / eps with
// the fixed eps = sqrt(machine epsilon) (jacobian_mf_op), the Krylov solver
// is GMRES without preconditioner (PCNONE), the step u <- u - alpha du takes
// the reference's line searches with non-finite trial residuals mapped to
// 1e100, and the stopping test |R| <= tau_abs is checked after every step
// (the solver never sets the relative tolerance's r0, so tau_rel has no
// effect). No Jacobian is stored.
extern "C" icx_status icx_mfnk_solve(icx_ctx* c, double* d_u, const icx_newton_options* opt, icx_newton_report* rep) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !opt) return set_err(c, ICX_ERR_INVALID, "null argument");
  if (opt->gmres_restart < 1 || opt->gmres_restart > 60) return set_err(c, ICX_ERR_INVALID, "restart in 1..60");
  cudaStream_t s = 0;
  icx_status st = ensure_work(c, opt->gmres_restart);
  if (st != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  const icx::DeviceMesh& dm = c->dm;
  const long long n = w->n;
  icx_newton_report local{};
  icx_newton_report* R = rep ? rep : &local;
  std::memset(R, 0, sizeof(*R));
  const double eps = std::sqrt(DBL_EPSILON);
  // w->res = R(u); w->ustep / w->rwork are the perturbed state and residual of
  // the Krylov products, w->z holds the line search's trial residual
  CK(icx::launch_residual(dm, c->phys, d_u, w->res, s));
  double rk = dev_norm(c, w->res, s);
  if (!std::isfinite(rk)) {
    SYNC_AT("initial residual");
    return set_err(c, ICX_ERR_NONFINITE, "non-finite initial residual");
  }
  R->r0 = rk;
  R->residual_history[0] = rk;
  icx::KrylovBuffers kb;
  kb.n = n;
  kb.m = opt->gmres_restart;
  kb.V = w->V;
  kb.w = w->w;
  kb.z = w->r;      // no preconditioner: gmres_op does not use z
  kb.r = w->rwork;  // restart residual
  kb.dh = w->dh;
  kb.lw = &w->lw;
  // the Krylov products need their own state/residual buffers: pct and du
  // are free while GMRES runs (du receives the solution at the end)
  double* up = w->pct;
  double* rp = w->ustep;
  icx::LinOp A = [&](const double* p, double* y, cudaStream_t st) -> cudaError_t {
    cudaError_t e = icx::la_xpay(n, d_u, eps, p, up, st);  // up = u + eps p
    if (e == cudaSuccess) e = icx::launch_residual(dm, c->phys, up, rp, st);
    if (e == cudaSuccess) e = icx::la_xpay(n, rp, -1.0, w->res, y, st);       // R(u + eps p) - R(u)
    if (e == cudaSuccess) e = icx::la_axpby(n, 1.0 / eps, y, 0.0, y, st);    // / eps
    return e;
  };
  bool converged = false;
  int k = 0;
  for (; k < opt->kmax; ++k) {
    int it = 0;
    double rr = 0.0;
    st = icx::gmres_op(kb, A, nullptr, opt->gmres_max_it, opt->gmres_rtol, w->res, w->du, &it, &rr, s, &c->err);
    if (st != ICX_OK) {
      SYNC_AT("linear solve");
      return st;
    }
    R->linear_iterations_total += it;
    double alpha = 1.0;
    if (opt->linesearch != 0) {
      std::function<double(double)> phi = [&](double a) -> double {
        icx::la_xpay(n, d_u, -a, w->du, w->ustep, s);
        icx::launch_residual(dm, c->phys, w->ustep, w->z, s);
        double v = dev_norm(c, w->z, s);
        return std::isfinite(v) ? v : 1e100;
      };
      if (opt->linesearch == 1)
        alpha = wolfe_ls(phi, opt->ls_alpha_max, opt->ls_alpha_initial, opt->ls_max_it, opt->ls_c1, opt->ls_c2);
      else
        alpha = corrigan_ls(phi, opt->ls_alpha_max, opt->ls_alpha_initial, opt->ls_max_it, opt->ls_alpha_min);
      SYNC_AT("line search");
    }
    CK(icx::la_axpby(n, -alpha, w->du, 1.0, d_u, s));
    CK(icx::launch_residual(dm, c->phys, d_u, w->res, s));
    rk = dev_norm(c, w->res, s);
    if (k + 1 < 64) {
      R->residual_history[k + 1] = rk;
      R->alpha_history[k] = alpha;
    }
    if (opt->verbosity > 0) std::printf("mfnk %d: |r| = %.6e alpha = %.4f gmres its = %d\n", k, rk, alpha, it);
    if (!std::isfinite(rk)) {
      SYNC_AT("residual");
      return set_err(c, ICX_ERR_NONFINITE, "non-finite residual");
    }
    if (rk <= opt->tau_abs) {
      converged = true;
      ++k;
      break;
    }
  }
  SYNC_AT("mfnk");
  R->iterations = k;
  R->converged = converged;
  R->r_final = rk;
  return converged ? ICX_OK : ICX_ERR_NOT_CONVERGED;
}

namespace icx {

icx_status solver_prepare_pc(icx_ctx* c, const double* vals, int kind, int sweeps) {
  icx_status st = ensure_work(c, 30);
  if (st != ICX_OK) return st;
  if ((st = ensure_mixed(c)) != ICX_OK) return st;
  icx_solver_work* w = c->sw;
  if (sweeps >= 0) w->sweeps = sweeps;  // negative: keep the solver's
  cudaStream_t s = 0;
  CK(cudaMemcpyAsync(w->vals, vals, sizeof(double) * (size_t)c->dm.nnzb * w->bs * w->bs, cudaMemcpyDeviceToDevice, s));
  CK(build_pc(c, kind, true, s));
  SYNC_AT("preconditioner");
  return ICX_OK;
}

cudaError_t solver_apply_pc(icx_ctx* c, int kind, bool mixed, const double* x, double* z, cudaStream_t s) {
  return apply_pc(c, kind, mixed, x, z, s);
}

const float* solver_vals32(icx_ctx* c) { return c->sw ? c->sw->vals32 : nullptr; }

cudaError_t solver_apply_ilu_flow(icx_ctx* c, bool mixed, const double* x, double* z, cudaStream_t s) {
  return ilu_flow(c, mixed, x, z, s);
}

// ---- the pieces a batch of independent solves drives per group context
icx_status solver_group_ready(icx_ctx* c, int precision, int pc_sweeps, int ilu_tile, bool graphs) {
  // one Krylov vector of the group's own: the batch holds the Krylov basis
  icx_status st = ensure_work(c, 1);
  if (st != ICX_OK) return st;
  if (precision >= 1 && (st = ensure_mixed(c)) != ICX_OK) return st;
  c->sw->sweeps = pc_sweeps;
  c->sw->graphs_on = graphs;
  if (ilu_tile >= 0) c->ilu_tile = ilu_tile;
  return ICX_OK;
}

cudaError_t solver_linearise(icx_ctx* c, const double* u, double* res, int precision, cudaStream_t s) {
  icx_solver_work* w = c->sw;
  if (precision != 2) return launch_jacobian_fd(c->dm, c->phys, u, res, w->vals, std::sqrt(DBL_EPSILON), s);
  cudaError_t e = launch_jacobian_fd_f32(c->dm, c->phys, u, res, w->vals32, s);
  return e == cudaSuccess ? la_f2d((long long)w->nnzb * w->bs * w->bs, w->vals32, w->vals, s) : e;
}

cudaError_t solver_build_pc(icx_ctx* c, int kind, bool mixed, cudaStream_t s) { return build_pc(c, kind, mixed, s); }

cudaError_t solver_operator(icx_ctx* c, bool mixed, const double* x, double* y, cudaStream_t s) {
  icx_solver_work* w = c->sw;
  return mixed ? launch_bsr_spmv_f32(c->dm, w->vals32, x, y, s) : launch_bsr_spmv(c->dm, w->vals, x, y, s);
}

const int* solver_flag(icx_ctx* c) { return c->sw ? c->sw->flag : nullptr; }

// whether preconditioner `pc` launches the same kernels with the same
// arguments at every apply (the condition of the Arnoldi-step graphs)
bool solver_graphable(icx_ctx* c, int pc, bool mixed) {
  icx_solver_work* w = c->sw;
  if (!w || !w->graphs_on) return false;
  if (pc == 0 || pc == 1 || pc == 3 || pc == 4) return true;
  if (pc == 5 && icx::lpc_zero_correction(c)) return solver_graphable(c, w->sweeps > 0 ? 4 : 2, mixed);
  if (pc != 2) return false;
  // the group apply and the sentinel schedule launch the same arguments every time
  const int pi = mixed ? 1 : 0;
  if (w->tp.tile && w->tp.group_ok && ilu_schedule(c->dm.tile, pi, true) >= 3) return true;
  return flow_sentinel(c->dm.tile, pi) && !(w->rows_ok && w->schedule == 2);
}

// what the launches of a preconditioner apply and operator product depend on
// (FNV-1a; a graph holding them is replayed only under the same key)
unsigned long long solver_graph_key(icx_ctx* c, int pc, bool mixed) {
  icx_solver_work* w = c->sw;
  const DeviceMesh& dm = c->dm;
  const TileChoice& t = dm.tile;
  const int pi = mixed ? 1 : 0;
  unsigned long long key = 1469598103934665603ull;
  for (long long v : {(long long)pc, (long long)mixed, (long long)w->sweeps, (long long)t.flow_rows[pi],
                      (long long)t.flow_ctas[pi], (long long)t.flow_sched[pi], (long long)(uintptr_t)dm.bsr_rowptr,
                      (long long)(uintptr_t)dm.bsr_colidx, (long long)(uintptr_t)dm.bsr_diag,
                      (long long)(uintptr_t)w->order, (long long)w->tp.tile, (long long)(uintptr_t)w->tp.order,
                      (long long)(uintptr_t)w->vals, (long long)(uintptr_t)w->pc})
    key = (key ^ (unsigned long long)v) * 1099511628211ull;
  return key;
}

double solver_line_search(int kind, const std::function<double(double)>& f, const icx_newton_options& o) {
  if (kind == 1) return wolfe_ls(f, o.ls_alpha_max, o.ls_alpha_initial, o.ls_max_it, o.ls_c1, o.ls_c2);
  if (kind == 2) return corrigan_ls(f, o.ls_alpha_max, o.ls_alpha_initial, o.ls_max_it, o.ls_alpha_min);
  return 1.0;
}

icx_status solver_take_pc_err(icx_ctx* c, int* err) {
  icx_solver_work* w = c->sw;
  cudaStream_t s = 0;
  *err = 0;
  CK(cudaMemcpyAsync(err, w->pc_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (*err) {
    // the counters are inconsistent after an abandoned apply: start over
    CK(cudaMemsetAsync(w->pc_err, 0, sizeof(int), s));
    CK(cudaMemsetAsync(w->cnt, 0, sizeof(unsigned) * 2 * c->dm.E, s));
    w->epoch = 0;
    CK(cudaStreamSynchronize(s));
  }
  return ICX_OK;
}

}  // namespace icx
