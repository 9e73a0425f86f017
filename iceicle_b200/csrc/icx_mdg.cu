// MDG-ICE on the GPU: node selection and parametrisation (geo_dof_map with
// hyper_rectangle, fe_function/geo_layouts.hpp:359-540), the interface
// conservation residual (ConservationLawDDG::interface_conservation,
// conservation_law.hpp:1178-1288; form_mdg_residual, form_residual.hpp:327-381),
// the Jacobian of [R; ICE] with respect to [u; x] (form_petsc_jacobian_fd +
// form_petsc_mdg_jacobian_fd, form_petsc_jacobian.hpp:55-317, 665-1049)
// assembled into CSR, and the regularised Gauss-Newton / Levenberg-Marquardt
// solver (CorriganLM, corrigan_lm.hpp:112-718, matrix-free subproblem
// corrigan_lm.hpp:68-109).
//
// Node-position derivatives move one node at a time, so the kernels evaluate
// element and face integrals with geometry computed on the fly from the
// (perturbed) node coordinates, one thread per (work item, perturbation).
// Boundary data and sources stay at their tabulated values while a node is
// perturbed (they are evaluated by host callbacks); the reference re-evaluates
// the callbacks at the moved points, which differs only where that data varies
// along a moving boundary.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <vector>

#include "icx_dg.cuh"
#include "icx_linalg.h"

struct icx_mdg_state {
  // selection (host)
  std::vector<int> traces;
  int hyper = 0;
  int nsel = 0, ngeo = 0;
  std::vector<int> sel, inv, fixmask, cols;
  std::vector<double> fixval;
  // device
  int* d_traces = nullptr;
  int* d_trace_nodes = nullptr;  // [ntr][g+1] selected index of each face node or nsel
  int* d_adj_ptr = nullptr;      // node -> (trace, local node) list
  int* d_adj = nullptr;
  double* d_psi = nullptr;       // [nqf][g+1] trace (geometry) basis at the face points
  double* d_rtr = nullptr;       // [ntr][(g+1)*neq] per-trace interface conservation
  int* d_fixmask = nullptr;
  double* d_fixval = nullptr;
  int* d_sel = nullptr;
  int* d_cols = nullptr;
  // Jacobian: work items and slots, CSR pattern of J and of J^T
  int nitems = 0;
  long long nslots = 0;
  int* d_items = nullptr;        // [nitems][6]
  double* d_slots = nullptr;
  long long nnz = 0;
  long long nrow = 0, ncol = 0;
  int* d_rowptr = nullptr;
  int* d_colidx = nullptr;
  int* d_src_ptr = nullptr;      // per CSR entry: range in d_src
  long long* d_src = nullptr;    // source index: < nbsr -> BSR value, else slot (index - nbsr)
  int* d_t_rowptr = nullptr;     // transpose
  int* d_t_colidx = nullptr;
  int* d_t_perm = nullptr;       // transpose position -> CSR position
  std::vector<int> h_rowptr, h_colidx;
  // LM buffers
  double* d_vals = nullptr;      // CSR values of J
  double* d_tvals = nullptr;     // CSR values of J^T
  double* d_bsr = nullptr;       // DG Jacobian blocks
  double* d_colnorm = nullptr;
  double* d_diag = nullptr;
  double* d_tmp = nullptr;       // length nrow
  double* d_res = nullptr;       // [res; ic]
  double* d_jtr = nullptr;
  double* d_p = nullptr;
  double* d_ustep = nullptr;
  double* d_rwork = nullptr;
  double* d_x = nullptr;         // current geometry parameters (device copy)
  double* d_colnorm2 = nullptr;  // length ncol: scratch of the subproblem ILU apply
  icx::KrylovBuffers kb;
  double* d_kV = nullptr;
  double* d_kw = nullptr;
  double* d_kz = nullptr;
  double* d_kr = nullptr;
  double* d_kdh = nullptr;
  icx::LinalgWork lw;
  std::vector<int> h_trowptr, h_tcolidx;  // transpose pattern (host)
  // explicitly formed LM subproblem A = J^T J + regularisation (CSR over the
  // unknowns [u; x]) and its scalar ILU(0), level-scheduled
  bool a_built = false;
  long long a_nnz = 0;
  int* d_a_rowptr = nullptr;
  int* d_a_colidx = nullptr;
  int* d_a_diag = nullptr;       // position of the diagonal entry of each row
  double* d_a_vals = nullptr;
  double* d_a_lu = nullptr;
  std::vector<int> lo_off, up_off;  // ILU levels: rows lo_rows[lo_off[l] .. lo_off[l + 1]) etc.
  int* d_lo_rows = nullptr;
  int* d_up_rows = nullptr;
  int* d_pc_err = nullptr;
  // data-flow triangular solves of the subproblem's ILU(0): per-row flags,
  // the two row counters of one apply, the wait-timeout flag, the last epoch
  unsigned* d_tri_ready = nullptr;
  unsigned* d_tri_next = nullptr;
  int* d_tri_err = nullptr;
  unsigned tri_epoch = 0;
  // Laplacian and element-wise regularisation: per element the pairs
  // (local node i, local node j, position in A) of free coordinates of two
  // selected nodes, and per touched position the pairs that add to it
  int npairs = 0, npos = 0;
  int* d_pair_ptr = nullptr;     // [E + 1]
  int* d_pair_ij = nullptr;      // [npairs][2]
  int* d_upos = nullptr;         // [npos] positions in A
  int* d_upos_ptr = nullptr;     // [npos + 1] into d_upos_list
  int* d_upos_list = nullptr;    // [npairs] pair indices, ascending
  double* d_pair_val = nullptr;  // [npairs]
  double* d_lam_el = nullptr;    // [E]
  double* d_cg_tab = nullptr;    // [(g+1)^2 points][ng][2] reference gradients + [points] weights
  double* d_detmin = nullptr;    // [E] minimum det J over the volume points
};

namespace icx {

// ------------------------------------------------------------- device part
template <int G>
struct GeoInline {
  static constexpr int NG = (G + 1) * (G + 1);
  // x, J, transformation Hessian at a tabulated point t ([NG][6])
  __device__ static void eval(const double* xn, const double* t, double x[2], double J[2][2], double H[2][3]) {
    x[0] = x[1] = 0.0;
    J[0][0] = J[0][1] = J[1][0] = J[1][1] = 0.0;
    H[0][0] = H[0][1] = H[0][2] = H[1][0] = H[1][1] = H[1][2] = 0.0;
    for (int n = 0; n < NG; ++n) {
      const double* tn = t + n * 6;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        double xv = xn[2 * n + i];
        x[i] += tn[0] * xv;
        J[i][0] += tn[1] * xv;
        J[i][1] += tn[2] * xv;
        H[i][0] += tn[3] * xv;
        H[i][1] += tn[4] * xv;
        H[i][2] += tn[5] * xv;
      }
    }
  }
  __device__ static void centroid(const DeviceMesh& dm, const double* xn, double c[2]) {
    c[0] = c[1] = 0.0;
    for (int n = 0; n < NG; ++n) {
      c[0] += dm.tab_gcen[n] * xn[2 * n];
      c[1] += dm.tab_gcen[n] * xn[2 * n + 1];
    }
  }
};

__device__ inline void jinv(const double J[2][2], double* Ji, double* det_out) {
  double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  double ds = (det == 0.0) ? 1.0 : det;
  Ji[0] = J[1][1] / ds;
  Ji[1] = -J[0][1] / ds;
  Ji[2] = -J[1][0] / ds;
  Ji[3] = J[0][0] / ds;
  if (det_out) *det_out = det;
}

__constant__ double c_mdg_dxi_ds[4][2] = {{0.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}};

template <int PDE, int P, int G>
struct MdgEval {
  using C = Cfg<PDE, P, G>;
  static constexpr int NEQ = C::NEQ, NB = C::NB, BS = C::BS, NQF = C::NQF, NQV = C::NQV, NG = C::NG;

  // domain_integral of element e (conservation_law.hpp:244-314), res += (BS)
  __device__ static void domain(const DeviceMesh& dm, const PhysParams& pp, int e, const double* xn, const double* ue,
                                double* res) {
    for (int q = 0; q < NQV; ++q) {
      double J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
      for (int n = 0; n < NG; ++n) {
        double d0 = dm.tab_gvol[(q * NG + n) * 2], d1 = dm.tab_gvol[(q * NG + n) * 2 + 1];
        J[0][0] += d0 * xn[2 * n]; J[0][1] += d1 * xn[2 * n];
        J[1][0] += d0 * xn[2 * n + 1]; J[1][1] += d1 * xn[2 * n + 1];
      }
      double Ji[4], det;
      jinv(J, Ji, &det);
      double wd = fmax(0.0, det) * dm.tab_vol[(size_t)NQV * NB * 3 + q];
      const double* tb = dm.tab_vol + (size_t)q * NB * 3;
      double u[NEQ], gxi[NEQ][2];
      for (int k = 0; k < NEQ; ++k) { u[k] = 0.0; gxi[k][0] = gxi[k][1] = 0.0; }
      for (int i = 0; i < NB; ++i)
        for (int k = 0; k < NEQ; ++k) {
          double c = ue[i * NEQ + k];
          u[k] += c * tb[i * 3];
          gxi[k][0] += c * tb[i * 3 + 1];
          gxi[k][1] += c * tb[i * 3 + 2];
        }
      double gx[2 * NEQ], F[2 * NEQ];
      for (int k = 0; k < NEQ; ++k)
        for (int d = 0; d < 2; ++d) gx[k * 2 + d] = gxi[k][0] * Ji[0 * 2 + d] + gxi[k][1] * Ji[1 * 2 + d];
      Phys<PDE>::flux(pp, u, gx, F);
      double Gq[NEQ][2];
      for (int k = 0; k < NEQ; ++k)
        for (int kk = 0; kk < 2; ++kk) Gq[k][kk] = (F[k * 2 + 0] * Ji[kk * 2 + 0] + F[k * 2 + 1] * Ji[kk * 2 + 1]) * wd;
      for (int i = 0; i < NB; ++i)
        for (int k = 0; k < NEQ; ++k) {
          double v = tb[i * 3 + 1] * Gq[k][0] + tb[i * 3 + 2] * Gq[k][1];
          if (dm.src) v -= dm.src[((size_t)e * NQV + q) * NEQ + k] * wd * tb[i * 3];
          res[i * NEQ + k] += v;
        }
    }
  }

  // geometry of face point q with both sides' node coordinates
  __device__ static void face_geo(const DeviceMesh& dm, const int* fi, const double* xL, const double* xR, int q,
                                  FacePt& fp, double x[2]) {
    int R = fi[1], fnl = fi[2], fnr = fi[3], orient = fi[4];
    double J[2][2], H[2][3];
    GeoInline<G>::eval(xL, dm.tab_gface + ((size_t)((fnl * 2 + 0) * NQF + q) * NG) * 6, x, J, H);
    double t0 = J[0][0] * c_mdg_dxi_ds[fnl][0] + J[0][1] * c_mdg_dxi_ds[fnl][1];
    double t1 = J[1][0] * c_mdg_dxi_ds[fnl][0] + J[1][1] * c_mdg_dxi_ds[fnl][1];
    double sqrtg = sqrt(t0 * t0 + t1 * t1);
    double nn = sqrt(t1 * t1 + t0 * t0);
    fp.n[0] = t1 / nn;
    fp.n[1] = -t0 / nn;
    fp.wsq = dm.qw_face[q] * sqrtg;
    jinv(J, fp.JiL, nullptr);
    for (int m = 0; m < 2; ++m)
      for (int a = 0; a < 3; ++a) fp.HL[3 * m + a] = H[m][a];
    double cL[2];
    GeoInline<G>::centroid(dm, xL, cL);
    double h;
    if (R >= 0) {
      double xr[2], JR[2][2], HR[2][3], cR[2];
      GeoInline<G>::eval(xR, dm.tab_gface + ((size_t)((fnr * 2 + orient) * NQF + q) * NG) * 6, xr, JR, HR);
      GeoInline<G>::centroid(dm, xR, cR);
      h = fp.n[0] * ((x[0] - cL[0]) + (cR[0] - x[0])) + fp.n[1] * ((x[1] - cL[1]) + (cR[1] - x[1]));
      jinv(JR, fp.JiR, nullptr);
      for (int m = 0; m < 2; ++m)
        for (int a = 0; a < 3; ++a) fp.HR[3 * m + a] = HR[m][a];
    } else {
      h = fabs(fp.n[0] * (x[0] - cL[0])) + fabs(fp.n[1] * (x[1] - cL[1]));
      for (int a = 0; a < 4; ++a) fp.JiR[a] = 0.0;
      for (int a = 0; a < 6; ++a) fp.HR[a] = 0.0;
    }
    fp.h = copysign(fmax(fabs(h), DBL_EPSILON), h);
  }

  // trace_integral / boundaryIntegral of face f: resL, resR += (BS each)
  template <bool DDG>
  __device__ static void trace(const DeviceMesh& dm, const PhysParams& pp, int f, const double* xL, const double* xR,
                               const double* uL, const double* uR, double* resL, double* resR) {
    const int* fi = dm.face_info + 8 * f;
    bool interior = fi[1] >= 0;
    const bool ic = Phys<PDE>::has_ic && pp.sigma_ic != 0.0;
    for (int q = 0; q < NQF; ++q) {
      FacePt fp;
      double x[2];
      face_geo(dm, fi, xL, xR, q, fp, x);
      const double* tL = dm.tab_face + (size_t)((fi[2] * 2 + 0) * NQF + q) * NB * 6;
      const double* tR = dm.tab_face + (size_t)((fi[3] * 2 + fi[4]) * NQF + q) * NB * 6;
      double sL[7 * NEQ], sR[7 * NEQ];
      side_state<NB, NEQ, DDG>(uL, tL, fp.JiL, fp.HL, sL, sL + NEQ, sL + 3 * NEQ);
      if (interior) side_state<NB, NEQ, DDG>(uR, tR, fp.JiR, fp.HR, sR, sR + NEQ, sR + 3 * NEQ);
      const double* bval = interior ? nullptr : dm.bvals + ((size_t)fi[7] * NQF + q) * NEQ;
      double out[NEQ], gq[4];
      face_flux_states<PDE, DDG>(pp, fp, interior, fi[5], bval, sL, sL + NEQ, sL + 3 * NEQ, sR, sR + NEQ,
                                 sR + 3 * NEQ, out, gq);
      for (int i = 0; i < NB; ++i)
        for (int k = 0; k < NEQ; ++k) {
          double v = out[k] * tL[i * 6];
          if (ic) v -= tL[i * 6 + 1] * gq[0] + tL[i * 6 + 2] * gq[1];
          resL[i * NEQ + k] += v;
        }
      if (interior)
        for (int i = 0; i < NB; ++i)
          for (int k = 0; k < NEQ; ++k) {
            double v = -out[k] * tR[i * 6];
            if (ic) v -= tR[i * 6 + 1] * gq[2] + tR[i * 6 + 2] * gq[3];
            resR[i * NEQ + k] += v;
          }
    }
  }

  // interface_conservation of face f: r[(G+1)*NEQ] (overwritten)
  __device__ static void ice(const DeviceMesh& dm, const PhysParams& pp, const double* psi, int f, const double* xL,
                             const double* xR, const double* uL, const double* uR, double* r) {
    const int* fi = dm.face_info + 8 * f;
    bool interior = fi[1] >= 0;
    for (int a = 0; a < (G + 1) * NEQ; ++a) r[a] = 0.0;
    if (!interior && fi[5] != ICX_BC_DIRICHLET) return;  // other boundary kinds: no interface condition
    for (int q = 0; q < NQF; ++q) {
      double x[2], J[2][2], H[2][3];
      int fnl = fi[2];
      GeoInline<G>::eval(xL, dm.tab_gface + ((size_t)((fnl * 2 + 0) * NQF + q) * NG) * 6, x, J, H);
      double t0 = J[0][0] * c_mdg_dxi_ds[fnl][0] + J[0][1] * c_mdg_dxi_ds[fnl][1];
      double t1 = J[1][0] * c_mdg_dxi_ds[fnl][0] + J[1][1] * c_mdg_dxi_ds[fnl][1];
      double sqrtg = sqrt(t0 * t0 + t1 * t1);
      double nn = sqrt(t1 * t1 + t0 * t0);
      double n[2] = {t1 / nn, -t0 / nn};
      double JiL[4], JiR[4];
      jinv(J, JiL, nullptr);
      // the right side of a boundary trace is the left element again, at its
      // local face 0 with orientation 0 (trace construction of the reference)
      int fr = interior ? fi[3] : 0, orr = interior ? fi[4] : 0;
      const double* xRn = interior ? xR : xL;
      {
        double xr[2], JR[2][2], HR[2][3];
        GeoInline<G>::eval(xRn, dm.tab_gface + ((size_t)((fr * 2 + orr) * NQF + q) * NG) * 6, xr, JR, HR);
        jinv(JR, JiR, nullptr);
      }
      double ul[NEQ], gl[2 * NEQ], hl[4 * NEQ], ur[NEQ], gr[2 * NEQ], hr[4 * NEQ];
      double Hz[6] = {0, 0, 0, 0, 0, 0};
      side_state<NB, NEQ, false>(uL, dm.tab_face + (size_t)((fnl * 2 + 0) * NQF + q) * NB * 6, JiL, Hz, ul, gl, hl);
      side_state<NB, NEQ, false>(interior ? uR : uL, dm.tab_face + (size_t)((fr * 2 + orr) * NQF + q) * NB * 6, JiR,
                                 Hz, ur, gr, hr);
      if (!interior)
        for (int k = 0; k < NEQ; ++k) ur[k] = dm.bvals[((size_t)fi[7] * NQF + q) * NEQ + k];
      if (P == 1)  // linear elements: gradients dropped (conservation_law.hpp:1262-1266)
        for (int k = 0; k < 2 * NEQ; ++k) gl[k] = gr[k] = 0.0;
      double FL[2 * NEQ], FR[2 * NEQ];
      Phys<PDE>::flux(pp, ul, gl, FL);
      Phys<PDE>::flux(pp, ur, gr, FR);
      for (int k = 0; k < NEQ; ++k) {
        double jump = (FR[k * 2] * n[0] + FR[k * 2 + 1] * n[1]) - (FL[k * 2] * n[0] + FL[k * 2 + 1] * n[1]);
        for (int i = 0; i <= G; ++i) r[i * NEQ + k] -= jump * sqrtg * dm.qw_face[q] * psi[q * (G + 1) + i];
      }
    }
  }
};

template <int G>
__device__ inline void load_nodes(const DeviceMesh& dm, int e, double* xn) {
  constexpr int NG = (G + 1) * (G + 1);
  for (int n = 0; n < NG; ++n) {
    int gn = dm.el_nodes[e * NG + n];
    xn[2 * n] = dm.coord[2 * gn];
    xn[2 * n + 1] = dm.coord[2 * gn + 1];
  }
}

// per selected trace: interface conservation r_t
template <int PDE, int P, int G>
__global__ void mdg_ice_trace_kernel(DeviceMesh dm, PhysParams pp, const double* __restrict__ u, int ntr,
                                     const int* __restrict__ traces, const double* __restrict__ psi,
                                     double* __restrict__ rtr) {
  using M = MdgEval<PDE, P, G>;
  constexpr int NG = (G + 1) * (G + 1);
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntr) return;
  int f = traces[t];
  const int* fi = dm.face_info + 8 * f;
  int L = fi[0], R = fi[1] >= 0 ? fi[1] : fi[0];
  double xL[2 * NG], xR[2 * NG];
  load_nodes<G>(dm, L, xL);
  load_nodes<G>(dm, R, xR);
  M::ice(dm, pp, psi, f, xL, xR, u + (size_t)L * M::BS, u + (size_t)R * M::BS, rtr + (size_t)t * (G + 1) * M::NEQ);
}

// per selected node and equation: ic = sum of the adjacent traces' entries
__global__ void mdg_ice_gather_kernel(int nsel, int neq, int g1, const int* __restrict__ adj_ptr,
                                      const int* __restrict__ adj, const double* __restrict__ rtr,
                                      double* __restrict__ ic) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nsel * neq) return;
  int k = t / neq, e = t - k * neq;
  double s = 0.0;
  for (int a = adj_ptr[k]; a < adj_ptr[k + 1]; ++a) {
    int tr = adj[2 * a], i = adj[2 * a + 1];
    s += rtr[((size_t)tr * g1 + i) * neq + e];
  }
  ic[t] = s;
}

// parameters of selected node k moved by de in component is: new coordinates
__device__ inline void node_perturbed(const int* fixmask, const double* fixval, int k, const double* cur, int is,
                                      double de, const double* box, double xy[2]) {
  int m = fixmask[k], c = 0;
  for (int d = 0; d < 2; ++d) {
    if (m & (1 << d)) {
      xy[d] = fixval[2 * k + d];
    } else {
      double v = cur[d] + (c == is ? de : 0.0);
      if (m) v = fmin(box[2 + d], fmax(box[d], v));
      xy[d] = v;
      ++c;
    }
  }
}

// Jacobian work items, one thread each; item = {type, k_or_t, obj, aux, slot, side}
//   type 0: dICE/du   trace t (obj), perturbed DOF aux of side `side`
//   type 1: dR/dx     node k, element obj (volume integral), component aux
//   type 2: dR/dx     node k, face obj (trace / boundary integral), component aux
//   type 3: dICE/dx   node k, selected trace index obj, component aux
struct MdgJacArgs {
  const double* u;
  const int* items;
  int nitems;
  double* slots;
  const int* traces;
  const int* fixmask;
  const double* fixval;
  const int* sel;
  const double* psi;
  double eps;
  double box[4];
};

template <int PDE, int P, int G, bool DDG>
__global__ void mdg_jac_kernel(DeviceMesh dm, PhysParams pp, MdgJacArgs a) {
  using M = MdgEval<PDE, P, G>;
  constexpr int NG = (G + 1) * (G + 1), BS = M::BS, NEQ = M::NEQ, NI = (G + 1) * M::NEQ;
  int it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= a.nitems) return;
  const int* d = a.items + 6 * it;
  int type = d[0];
  double* out = a.slots + d[4];
  if (type == 0) {
    int f = a.traces[d[2]];
    const int* fi = dm.face_info + 8 * f;
    int L = fi[0], R = fi[1] >= 0 ? fi[1] : fi[0];
    double xL[2 * NG], xR[2 * NG], uL[BS], uR[BS], r0[NI], r1[NI];
    load_nodes<G>(dm, L, xL);
    load_nodes<G>(dm, R, xR);
    for (int i = 0; i < BS; ++i) { uL[i] = a.u[(size_t)L * BS + i]; uR[i] = a.u[(size_t)R * BS + i]; }
    M::ice(dm, pp, a.psi, f, xL, xR, uL, uR, r0);
    double nrm = 0.0;
    for (int i = 0; i < NI; ++i) nrm += r0[i] * r0[i];
    double es = fmax(a.eps, sqrt(nrm) * a.eps);
    if (d[5] == 0) uL[d[3]] += es; else uR[d[3]] += es;
    M::ice(dm, pp, a.psi, f, xL, xR, uL, uR, r1);
    for (int i = 0; i < NI; ++i) out[i] = (r1[i] - r0[i]) / es;
    return;
  }
  int k = d[1], node = a.sel[k], is = d[3];
  double cur[2] = {dm.coord[2 * node], dm.coord[2 * node + 1]};
  if (type == 1) {
    int e = d[2];
    double xn[2 * NG], r0[BS], r1[BS], ue[BS];
    load_nodes<G>(dm, e, xn);
    for (int i = 0; i < BS; ++i) { ue[i] = a.u[(size_t)e * BS + i]; r0[i] = 0.0; r1[i] = 0.0; }
    M::domain(dm, pp, e, xn, ue, r0);
    double nrm = 0.0;
    for (int i = 0; i < BS; ++i) nrm += r0[i] * r0[i];
    double es = fmax(a.eps, sqrt(nrm) * a.eps);
    double xy[2];
    node_perturbed(a.fixmask, a.fixval, k, cur, is, es, a.box, xy);
    for (int n = 0; n < NG; ++n)
      if (dm.el_nodes[e * NG + n] == node) { xn[2 * n] = xy[0]; xn[2 * n + 1] = xy[1]; }
    M::domain(dm, pp, e, xn, ue, r1);
    for (int i = 0; i < BS; ++i) out[i] = (r1[i] - r0[i]) / es;
    return;
  }
  if (type == 2) {
    int f = d[2];
    const int* fi = dm.face_info + 8 * f;
    int L = fi[0], R = fi[1];
    bool interior = R >= 0;
    double xL[2 * NG], xR[2 * NG], uL[BS], uR[BS], rl0[BS], rr0[BS], rl1[BS], rr1[BS];
    load_nodes<G>(dm, L, xL);
    load_nodes<G>(dm, interior ? R : L, xR);
    for (int i = 0; i < BS; ++i) {
      uL[i] = a.u[(size_t)L * BS + i];
      uR[i] = a.u[(size_t)(interior ? R : L) * BS + i];
      rl0[i] = rr0[i] = rl1[i] = rr1[i] = 0.0;
    }
    M::template trace<DDG>(dm, pp, f, xL, xR, uL, uR, rl0, rr0);
    double nl = 0.0, nr = 0.0;
    for (int i = 0; i < BS; ++i) { nl += rl0[i] * rl0[i]; nr += rr0[i] * rr0[i]; }
    double es = fmax(a.eps, fmax(sqrt(nl), sqrt(nr)) * a.eps);
    double xy[2];
    node_perturbed(a.fixmask, a.fixval, k, cur, is, es, a.box, xy);
    for (int n = 0; n < NG; ++n) {
      if (dm.el_nodes[L * NG + n] == node) { xL[2 * n] = xy[0]; xL[2 * n + 1] = xy[1]; }
      if (interior && dm.el_nodes[R * NG + n] == node) { xR[2 * n] = xy[0]; xR[2 * n + 1] = xy[1]; }
    }
    if (!interior)
      for (int n = 0; n < 2 * NG; ++n) xR[n] = xL[n];
    M::template trace<DDG>(dm, pp, f, xL, xR, uL, uR, rl1, rr1);
    for (int i = 0; i < BS; ++i) out[i] = (rl1[i] - rl0[i]) / es;
    for (int i = 0; i < BS; ++i) out[BS + i] = interior ? (rr1[i] - rr0[i]) / es : 0.0;
    return;
  }
  // type 3
  {
    int f = a.traces[d[2]];
    const int* fi = dm.face_info + 8 * f;
    int L = fi[0], R = fi[1] >= 0 ? fi[1] : fi[0];
    double xL[2 * NG], xR[2 * NG], uL[BS], uR[BS], r0[NI], r1[NI];
    load_nodes<G>(dm, L, xL);
    load_nodes<G>(dm, R, xR);
    for (int i = 0; i < BS; ++i) { uL[i] = a.u[(size_t)L * BS + i]; uR[i] = a.u[(size_t)R * BS + i]; }
    M::ice(dm, pp, a.psi, f, xL, xR, uL, uR, r0);
    double nrm = 0.0;
    for (int i = 0; i < NI; ++i) nrm += r0[i] * r0[i];
    double es = fmax(a.eps, sqrt(nrm) * a.eps);
    double xy[2];
    node_perturbed(a.fixmask, a.fixval, k, cur, is, es, a.box, xy);
    for (int n = 0; n < NG; ++n) {
      if (dm.el_nodes[L * NG + n] == node) { xL[2 * n] = xy[0]; xL[2 * n + 1] = xy[1]; }
      if (dm.el_nodes[R * NG + n] == node) { xR[2 * n] = xy[0]; xR[2 * n + 1] = xy[1]; }
    }
    M::ice(dm, pp, a.psi, f, xL, xR, uL, uR, r1);
    for (int i = 0; i < NI; ++i) out[i] = (r1[i] - r0[i]) / es;
  }
}

// CSR value assembly: vals[p] = sum of the sources of entry p
__global__ void mdg_assemble_kernel(long long nnz, const int* __restrict__ src_ptr, const long long* __restrict__ src,
                                    long long nbsr, const double* __restrict__ bsr, const double* __restrict__ slots,
                                    double* __restrict__ vals) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  double s = 0.0;
  for (int a = src_ptr[p]; a < src_ptr[p + 1]; ++a) {
    long long q = src[a];
    s += q < nbsr ? bsr[q] : slots[q - nbsr];
  }
  vals[p] = s;
}

__global__ void gather_kernel(long long n, const int* __restrict__ perm, const double* __restrict__ src,
                              double* __restrict__ dst) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) dst[p] = src[perm[p]];
}

// y = A x for CSR A, one warp per row
__global__ void csr_spmv_kernel(long long nrow, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
  long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (row >= nrow) return;
  double s = 0.0;
  for (int k = rowptr[row] + lane; k < rowptr[row + 1]; k += 32) s += vals[k] * x[colidx[k]];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) y[row] = s;
}

// row 2-norms of CSR A
__global__ void csr_rownorm_kernel(long long nrow, const int* __restrict__ rowptr, const double* __restrict__ vals,
                                   double* __restrict__ out) {
  long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (row >= nrow) return;
  double s = 0.0;
  for (int k = rowptr[row] + lane; k < rowptr[row + 1]; k += 32) s += vals[k] * vals[k];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) out[row] = sqrt(s);
}

// LM diagonal: lambda_u * colnorm (PDE unknowns), max(lambda_b, lambda_b * colnorm) (geometry)
__global__ void lm_diag_kernel(long long n, long long npde, double lu, double lb, const double* __restrict__ cn,
                               double* __restrict__ dgl) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dgl[i] = i < npde ? lu * cn[i] : fmax(lb, lb * cn[i]);
}

// y += d .* x
__global__ void diag_axpy_kernel(long long n, const double* __restrict__ dgl, const double* __restrict__ x,
                                 double* __restrict__ y) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += dgl[i] * x[i];
}

// ------------------------------------------------------------ dispatch
template <int PDE, int P, int G>
static cudaError_t ice_pg(const DeviceMesh& dm, const PhysParams& pp, const icx_mdg_state& m, const double* u,
                          double* ic, cudaStream_t s) {
  int ntr = (int)m.traces.size();
  if (ntr) mdg_ice_trace_kernel<PDE, P, G><<<(ntr + 127) / 128, 128, 0, s>>>(dm, pp, u, ntr, m.d_traces, m.d_psi,
                                                                           m.d_rtr);
  int n = m.nsel * dm.neq;
  if (n) mdg_ice_gather_kernel<<<(n + 127) / 128, 128, 0, s>>>(m.nsel, dm.neq, G + 1, m.d_adj_ptr, m.d_adj, m.d_rtr,
                                                                ic);
  return cudaGetLastError();
}

template <int PDE, int P, int G>
static cudaError_t mdgjac_pg(const DeviceMesh& dm, const PhysParams& pp, const MdgJacArgs& a, cudaStream_t s) {
  if (!a.nitems) return cudaSuccess;
  if (pp.beta1 != 0.0)
    mdg_jac_kernel<PDE, P, G, true><<<(a.nitems + 63) / 64, 64, 0, s>>>(dm, pp, a);
  else
    mdg_jac_kernel<PDE, P, G, false><<<(a.nitems + 63) / 64, 64, 0, s>>>(dm, pp, a);
  return cudaGetLastError();
}

#define ICX_MDG_DISPATCH(FN, ...)                                                              \
  do {                                                                                         \
    if (pp.pde == 0 && dm.P == 1 && dm.G == 1) return FN<0, 1, 1>(__VA_ARGS__);               \
    if (pp.pde == 0 && dm.P == 2 && dm.G == 1) return FN<0, 2, 1>(__VA_ARGS__);               \
    if (pp.pde == 0 && dm.P == 3 && dm.G == 1) return FN<0, 3, 1>(__VA_ARGS__);               \
    if (pp.pde == 0 && dm.P == 1 && dm.G == 2) return FN<0, 1, 2>(__VA_ARGS__);               \
    if (pp.pde == 0 && dm.P == 2 && dm.G == 2) return FN<0, 2, 2>(__VA_ARGS__);               \
    if (pp.pde == 1 && dm.P == 1 && dm.G == 1) return FN<1, 1, 1>(__VA_ARGS__);               \
    if (pp.pde == 1 && dm.P == 2 && dm.G == 1) return FN<1, 2, 1>(__VA_ARGS__);               \
    if (pp.pde == 1 && dm.P == 1 && dm.G == 2) return FN<1, 1, 2>(__VA_ARGS__);               \
    if (pp.pde == 1 && dm.P == 2 && dm.G == 2) return FN<1, 2, 2>(__VA_ARGS__);               \
    return cudaErrorInvalidValue;                                                              \
  } while (0)

static cudaError_t launch_ice(const DeviceMesh& dm, const PhysParams& pp, const icx_mdg_state& m, const double* u,
                              double* ic, cudaStream_t s) {
  ICX_MDG_DISPATCH(ice_pg, dm, pp, m, u, ic, s);
}

static cudaError_t launch_mdgjac(const DeviceMesh& dm, const PhysParams& pp, const MdgJacArgs& a, cudaStream_t s) {
  ICX_MDG_DISPATCH(mdgjac_pg, dm, pp, a, s);
}

void free_mdg(icx_ctx* c) {
  if (!c || !c->mdg) return;
  icx_mdg_state* m = c->mdg;
  void* ptrs[] = {m->d_traces, m->d_trace_nodes, m->d_adj_ptr, m->d_adj, m->d_psi, m->d_rtr, m->d_fixmask,
                  m->d_fixval, m->d_sel, m->d_cols, m->d_items, m->d_slots, m->d_rowptr, m->d_colidx,
                  m->d_src_ptr, m->d_src, m->d_t_rowptr, m->d_t_colidx, m->d_t_perm, m->d_vals, m->d_tvals,
                  m->d_bsr, m->d_colnorm, m->d_diag, m->d_tmp, m->d_res, m->d_jtr, m->d_p, m->d_ustep,
                  m->d_rwork, m->d_x, m->d_kV, m->d_kw, m->d_kz, m->d_kr, m->d_kdh, m->lw.partial,
                  m->d_a_rowptr, m->d_a_colidx, m->d_a_diag, m->d_a_vals, m->d_a_lu, m->d_lo_rows, m->d_up_rows,
                  m->d_pc_err, m->d_pair_ptr, m->d_pair_ij, m->d_upos, m->d_upos_ptr, m->d_upos_list,
                  m->d_pair_val, m->d_lam_el, m->d_cg_tab, m->d_detmin, m->d_colnorm2, m->d_tri_ready,
                  m->d_tri_next, m->d_tri_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete m;
  c->mdg = nullptr;
}

}  // namespace icx

// ------------------------------------------------------------------ host
namespace {

icx_status merr(icx_ctx* c, icx_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

#define MCK(expr)                                                                            \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess) return merr(c, ICX_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <class T>
cudaError_t up(T** d, const std::vector<T>& h) {
  if (*d) { cudaFree(*d); *d = nullptr; }
  if (h.empty()) return cudaSuccess;
  cudaError_t e = cudaMalloc((void**)d, sizeof(T) * h.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
}

// global node of face node i (geometry order g, s_i = -1 + 2 i / g along the left face)
int face_node(const icx_ctx* c, int f, int i) {
  const int* F = &c->faces[7 * f];
  int g = c->geo_order;
  double s = -1.0 + 2.0 * i / g, xi[2];
  switch (F[2]) {
    case 0: xi[0] = -1.0; xi[1] = -s; break;
    case 1: xi[0] = s; xi[1] = -1.0; break;
    case 2: xi[0] = 1.0; xi[1] = s; break;
    default: xi[0] = -s; xi[1] = 1.0; break;
  }
  int k0 = (int)std::lround((xi[0] + 1.0) * 0.5 * g), k1 = (int)std::lround((xi[1] + 1.0) * 0.5 * g);
  return c->el_nodes[(size_t)F[0] * (g + 1) * (g + 1) + k0 * (g + 1) + k1];
}

// parameters -> coordinates of the selected nodes (update_mesh, component_span.hpp:193-210)
void apply_x(icx_ctx* c, const double* x) {
  icx_mdg_state& m = *c->mdg;
  for (int k = 0; k < m.nsel; ++k) {
    int n = m.sel[k], cc = m.cols[k];
    for (int d = 0; d < 2; ++d) {
      if (m.fixmask[k] & (1 << d)) {
        c->coord[2 * n + d] = m.fixval[2 * k + d];
      } else {
        double v = x[cc++];
        if (m.fixmask[k]) v = std::min(d == 0 ? c->xmax[0] : c->xmax[1], std::max(d == 0 ? c->xmin[0] : c->xmin[1], v));
        c->coord[2 * n + d] = v;
      }
    }
  }
}

}  // namespace

extern "C" {

icx_status icx_mdg_select(icx_ctx* c, int ntraces, const int* traces, int hyper_rectangle) {
  if (c && !c->parts.empty()) return merr(c, ICX_ERR_UNSUPPORTED, "MDG-ICE on a batch of problems");
  if (!c || !c->ready) return merr(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (ntraces < 0 || (ntraces && !traces)) return merr(c, ICX_ERR_INVALID, "bad trace list");
  const icx::DeviceMesh& dm = c->dm;
  if (!((c->phys.pde == 0 && c->p <= 3 && c->geo_order <= 2) || (c->phys.pde == 1 && c->p <= 2 && c->geo_order <= 2)))
    return merr(c, ICX_ERR_UNSUPPORTED, "MDG-ICE kernels are built for Burgers p<=3 and Navier-Stokes p<=2");
  for (int t = 0; t < ntraces; ++t)
    if (traces[t] < 0 || traces[t] >= dm.F) return merr(c, ICX_ERR_INVALID, "trace index out of range");
  cudaSetDevice(c->device);
  icx::free_mdg(c);
  c->mdg = new icx_mdg_state();
  icx_mdg_state& m = *c->mdg;
  m.traces.assign(traces, traces + ntraces);
  m.hyper = hyper_rectangle;
  int g = c->geo_order, nn = dm.n_nodes;
  std::vector<char> pick(nn, 0);
  for (int t : m.traces)
    for (int i = 0; i <= g; ++i) pick[face_node(c, t, i)] = 1;
  for (int n = 0; n < nn; ++n)
    if (pick[n]) m.sel.push_back(n);
  m.nsel = (int)m.sel.size();
  m.inv.assign(nn, m.nsel);
  for (int k = 0; k < m.nsel; ++k) m.inv[m.sel[k]] = k;
  m.fixmask.assign(m.nsel, 0);
  m.fixval.assign(2 * m.nsel, 0.0);
  m.cols.assign(m.nsel + 1, 0);
  for (int k = 0; k < m.nsel; ++k) {
    int n = m.sel[k], mk = 0;
    // hyper_rectangle walks the (nx+1) x (ny+1) index product with a running
    // node counter (geo_layouts.hpp:520-537): on geometry-order-1 meshes this is
    // the node numbering itself
    if (hyper_rectangle && n < (c->nx + 1) * (c->ny + 1)) {
      int ix = n % (c->nx + 1), iy = n / (c->nx + 1);
      if (ix == 0) { mk |= 1; m.fixval[2 * k] = c->xmin[0]; }
      else if (ix == c->nx) { mk |= 1; m.fixval[2 * k] = c->xmax[0]; }
      if (iy == 0) { mk |= 2; m.fixval[2 * k + 1] = c->xmin[1]; }
      else if (iy == c->ny) { mk |= 2; m.fixval[2 * k + 1] = c->xmax[1]; }
    }
    m.fixmask[k] = mk;
    m.cols[k + 1] = m.cols[k] + 2 - ((mk & 1) ? 1 : 0) - ((mk & 2) ? 1 : 0);
  }
  m.ngeo = m.cols[m.nsel];
  // trace -> node adjacency for the interface-conservation gather
  std::vector<std::vector<std::pair<int, int>>> adj(m.nsel);
  for (int t = 0; t < ntraces; ++t)
    for (int i = 0; i <= g; ++i) {
      int k = m.inv[face_node(c, m.traces[t], i)];
      if (k < m.nsel) adj[k].push_back({t, i});
    }
  std::vector<int> aptr(m.nsel + 1, 0), alist;
  for (int k = 0; k < m.nsel; ++k) {
    for (auto& pr : adj[k]) { alist.push_back(pr.first); alist.push_back(pr.second); }
    aptr[k + 1] = (int)alist.size() / 2;
  }
  // trace basis at the face points
  double qx[16], qw[16];
  icx::gauss_legendre_points(dm.nqf, qx, qw);
  std::vector<double> psi((size_t)dm.nqf * (g + 1));
  for (int q = 0; q < dm.nqf; ++q) icx::lagrange_values(g, qx[q], &psi[(size_t)q * (g + 1)]);
  MCK(up(&m.d_traces, m.traces));
  MCK(up(&m.d_adj_ptr, aptr));
  MCK(up(&m.d_adj, alist));
  MCK(up(&m.d_psi, psi));
  MCK(up(&m.d_fixmask, m.fixmask));
  MCK(up(&m.d_fixval, m.fixval));
  MCK(up(&m.d_sel, m.sel));
  MCK(up(&m.d_cols, m.cols));
  if (ntraces) MCK(cudaMalloc((void**)&m.d_rtr, sizeof(double) * ntraces * (g + 1) * dm.neq));
  return ICX_OK;
}

icx_status icx_mdg_info(const icx_ctx* c, int* n_selected_nodes, int* n_geo) {
  if (!c || !c->mdg) return ICX_ERR_INVALID;
  if (n_selected_nodes) *n_selected_nodes = c->mdg->nsel;
  if (n_geo) *n_geo = c->mdg->ngeo;
  return ICX_OK;
}

icx_status icx_mdg_selected_nodes(const icx_ctx* c, int* nodes) {
  if (!c || !c->mdg || !nodes) return ICX_ERR_INVALID;
  std::memcpy(nodes, c->mdg->sel.data(), sizeof(int) * c->mdg->nsel);
  return ICX_OK;
}

icx_status icx_mdg_get_x(const icx_ctx* c, double* x) {
  if (!c || !c->mdg || !x) return ICX_ERR_INVALID;
  const icx_mdg_state& m = *c->mdg;
  for (int k = 0; k < m.nsel; ++k) {
    int n = m.sel[k], cc = m.cols[k];
    for (int d = 0; d < 2; ++d)
      if (!(m.fixmask[k] & (1 << d))) x[cc++] = c->coord[2 * n + d];
  }
  return ICX_OK;
}

icx_status icx_mdg_set_x(icx_ctx* c, const double* x) {
  if (!c || !c->mdg || !x) return merr(c, ICX_ERR_INVALID, "MDG selection missing");
  cudaSetDevice(c->device);
  apply_x(c, x);
  return icx::refresh_geometry(c);
}

icx_status icx_form_mdg_residual(icx_ctx* c, const double* d_u, double* d_ic, void* stream) {
  if (!c || !c->mdg) return merr(c, ICX_ERR_INVALID, "MDG selection missing");
  cudaError_t e = icx::launch_ice(c->dm, c->phys, *c->mdg, d_u, d_ic, (cudaStream_t)stream);
  if (e != cudaSuccess) return merr(c, ICX_ERR_CUDA, std::string("ice kernels: ") + cudaGetErrorString(e));
  return ICX_OK;
}

icx_status icx_form_residual_mdg(icx_ctx* c, const double* d_u, const double* x, double* d_res, double* d_ic,
                                 void* stream) {
  if (!c || !c->mdg) return merr(c, ICX_ERR_INVALID, "MDG selection missing");
  if (x) {
    icx_status st = icx_mdg_set_x(c, x);
    if (st != ICX_OK) return st;
  }
  icx_status st = icx_form_residual(c, d_u, d_res, stream);
  if (st != ICX_OK) return st;
  return icx_form_mdg_residual(c, d_u, d_ic, stream);
}

}  // extern "C"

// --------------------------------------------------- Jacobian pattern
namespace {

// builds work items, slot rows/cols and the CSR pattern of the full Jacobian
icx_status build_mdg_pattern(icx_ctx* c) {
  icx_mdg_state& m = *c->mdg;
  const icx::DeviceMesh& dm = c->dm;
  int g = c->geo_order, bs = dm.nb * dm.neq, neq = dm.neq, ni = (g + 1) * neq;
  long long N = (long long)dm.E * bs;
  m.nrow = N + (long long)m.nsel * neq;
  m.ncol = N + m.ngeo;
  std::vector<int> items;
  std::vector<long long> srow, scol;
  long long slot = 0;
  auto add_item = [&](int type, int k, int obj, int aux, int side, int nvals) {
    int rec[6] = {type, k, obj, aux, (int)slot, side};
    items.insert(items.end(), rec, rec + 6);
    slot += nvals;
  };
  auto ice_rows = [&](int t, long long col) {
    for (int i = 0; i <= g; ++i) {
      int kk = m.inv[face_node(c, m.traces[t], i)];
      for (int e = 0; e < neq; ++e) {
        srow.push_back(kk < m.nsel ? N + (long long)kk * neq + e : -1);
        scol.push_back(col);
      }
    }
  };
  // dICE/du
  for (int t = 0; t < (int)m.traces.size(); ++t) {
    const int* F = &c->faces[7 * m.traces[t]];
    int L = F[0], R = F[1] >= 0 ? F[1] : F[0];
    for (int side = 0; side < 2; ++side)
      for (int cdof = 0; cdof < bs; ++cdof) {
        add_item(0, 0, t, cdof, side, ni);
        ice_rows(t, (long long)(side ? R : L) * bs + cdof);
      }
  }
  // node stencils
  int ngl = (g + 1) * (g + 1);
  std::vector<std::vector<int>> el_of_node(dm.n_nodes);
  for (int e = 0; e < dm.E; ++e)
    for (int n = 0; n < ngl; ++n) el_of_node[c->el_nodes[(size_t)e * ngl + n]].push_back(e);
  std::vector<std::vector<int>> faces_of_el(dm.E);
  for (int f = 0; f < dm.F; ++f) {
    faces_of_el[c->faces[7 * f]].push_back(f);
    if (c->faces[7 * f + 1] >= 0) faces_of_el[c->faces[7 * f + 1]].push_back(f);
  }
  std::vector<int> tsel(dm.F, -1);
  for (int t = 0; t < (int)m.traces.size(); ++t) tsel[m.traces[t]] = t;
  for (int k = 0; k < m.nsel; ++k) {
    int node = m.sel[k], ns = m.cols[k + 1] - m.cols[k];
    if (!ns) continue;
    std::vector<int> els = el_of_node[node];
    std::sort(els.begin(), els.end());
    els.erase(std::unique(els.begin(), els.end()), els.end());
    std::vector<int> fv;
    for (int e : els)
      for (int f : faces_of_el[e]) fv.push_back(f);
    std::sort(fv.begin(), fv.end());
    fv.erase(std::unique(fv.begin(), fv.end()), fv.end());
    for (int is = 0; is < ns; ++is) {
      long long col = N + m.cols[k] + is;
      for (int e : els) {
        add_item(1, k, e, is, 0, bs);
        for (int i = 0; i < bs; ++i) { srow.push_back((long long)e * bs + i); scol.push_back(col); }
      }
      for (int f : fv) {
        int L = c->faces[7 * f], R = c->faces[7 * f + 1];
        add_item(2, k, f, is, 0, 2 * bs);
        for (int i = 0; i < bs; ++i) { srow.push_back((long long)L * bs + i); scol.push_back(col); }
        for (int i = 0; i < bs; ++i) { srow.push_back(R >= 0 ? (long long)R * bs + i : -1); scol.push_back(col); }
      }
      for (int f : fv) {
        if (tsel[f] < 0) continue;
        add_item(3, k, tsel[f], is, 0, ni);
        ice_rows(tsel[f], col);
      }
    }
  }
  m.nitems = (int)items.size() / 6;
  m.nslots = slot;
  // entries: (row, col, source)
  long long nbsr = (long long)dm.nnzb * bs * bs;
  std::vector<int> rowptr_b(dm.E + 1), colidx_b(dm.nnzb);
  cudaMemcpy(rowptr_b.data(), dm.bsr_rowptr, sizeof(int) * (dm.E + 1), cudaMemcpyDeviceToHost);
  cudaMemcpy(colidx_b.data(), dm.bsr_colidx, sizeof(int) * dm.nnzb, cudaMemcpyDeviceToHost);
  struct Ent { long long row, col, src; };
  std::vector<Ent> ent;
  ent.reserve(nbsr + slot);
  for (int r = 0; r < dm.E; ++r)
    for (int kb = rowptr_b[r]; kb < rowptr_b[r + 1]; ++kb)
      for (int i = 0; i < bs; ++i)
        for (int j = 0; j < bs; ++j)
          ent.push_back({(long long)r * bs + i, (long long)colidx_b[kb] * bs + j, ((long long)kb * bs + i) * bs + j});
  for (long long sidx = 0; sidx < slot; ++sidx)
    if (srow[sidx] >= 0) ent.push_back({srow[sidx], scol[sidx], nbsr + sidx});
  std::sort(ent.begin(), ent.end(), [](const Ent& a, const Ent& b) {
    return a.row != b.row ? a.row < b.row : (a.col != b.col ? a.col < b.col : a.src < b.src);
  });
  std::vector<int> rowptr(m.nrow + 1, 0), colidx, src_ptr(1, 0);
  std::vector<long long> src;
  src.reserve(ent.size());
  for (size_t a = 0; a < ent.size(); ++a) {
    if (a == 0 || ent[a].row != ent[a - 1].row || ent[a].col != ent[a - 1].col) {
      if (a) src_ptr.push_back((int)src.size());
      colidx.push_back((int)ent[a].col);
      rowptr[ent[a].row + 1]++;
    }
    src.push_back(ent[a].src);
  }
  src_ptr.push_back((int)src.size());
  for (long long r = 0; r < m.nrow; ++r) rowptr[r + 1] += rowptr[r];
  m.nnz = (long long)colidx.size();
  // transpose pattern
  std::vector<int> trow(m.ncol + 1, 0), tcol(m.nnz), tperm(m.nnz);
  for (long long p = 0; p < m.nnz; ++p) trow[colidx[p] + 1]++;
  for (long long cc = 0; cc < m.ncol; ++cc) trow[cc + 1] += trow[cc];
  std::vector<int> fill(trow.begin(), trow.end() - 1);
  for (long long r = 0; r < m.nrow; ++r)
    for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) {
      int q = fill[colidx[p]]++;
      tcol[q] = (int)r;
      tperm[q] = p;
    }
  m.h_rowptr = rowptr;
  m.h_colidx = colidx;
  m.h_trowptr = trow;
  m.h_tcolidx = tcol;
  m.a_built = false;
  MCK(up(&m.d_items, items));
  if (m.d_slots) cudaFree(m.d_slots);
  MCK(cudaMalloc((void**)&m.d_slots, sizeof(double) * std::max(slot, 1LL)));
  MCK(up(&m.d_rowptr, rowptr));
  MCK(up(&m.d_colidx, colidx));
  MCK(up(&m.d_src_ptr, src_ptr));
  MCK(up(&m.d_src, src));
  MCK(up(&m.d_t_rowptr, trow));
  MCK(up(&m.d_t_colidx, tcol));
  MCK(up(&m.d_t_perm, tperm));
  MCK(cudaMalloc((void**)&m.d_bsr, sizeof(double) * nbsr));
  MCK(cudaMalloc((void**)&m.d_vals, sizeof(double) * m.nnz));
  MCK(cudaMalloc((void**)&m.d_tvals, sizeof(double) * m.nnz));
  return ICX_OK;
}

}  // namespace

extern "C" {

icx_status icx_mdg_jacobian_pattern(icx_ctx* c, long long* nrow, long long* ncol, long long* nnz, int* rowptr,
                                    int* colidx) {
  if (!c || !c->mdg) return merr(c, ICX_ERR_INVALID, "MDG selection missing");
  if (!c->mdg->d_rowptr) {
    icx_status st = build_mdg_pattern(c);
    if (st != ICX_OK) return st;
  }
  icx_mdg_state& m = *c->mdg;
  if (nrow) *nrow = m.nrow;
  if (ncol) *ncol = m.ncol;
  if (nnz) *nnz = m.nnz;
  if (rowptr) std::memcpy(rowptr, m.h_rowptr.data(), sizeof(int) * (m.nrow + 1));
  if (colidx) std::memcpy(colidx, m.h_colidx.data(), sizeof(int) * m.nnz);
  return ICX_OK;
}

// [res; ic] and the CSR values of d[res; ic]/d[u; x] at the current mesh
icx_status icx_form_jacobian_mdg_fd(icx_ctx* c, const double* d_u, double* d_res, double* d_ic, double* d_csr_vals,
                                    double eps, void* stream) {
  if (!c || !c->mdg) return merr(c, ICX_ERR_INVALID, "MDG selection missing");
  icx_mdg_state& m = *c->mdg;
  if (!m.d_rowptr) {
    icx_status st = build_mdg_pattern(c);
    if (st != ICX_OK) return st;
  }
  if (!(eps > 0.0)) eps = std::sqrt(DBL_EPSILON);
  cudaStream_t s = (cudaStream_t)stream;
  const icx::DeviceMesh& dm = c->dm;
  MCK(icx::launch_jacobian_fd(dm, c->phys, d_u, d_res, m.d_bsr, eps, s));
  MCK(icx::launch_ice(dm, c->phys, m, d_u, d_ic, s));
  icx::MdgJacArgs a;
  a.u = d_u;
  a.items = m.d_items;
  a.nitems = m.nitems;
  a.slots = m.d_slots;
  a.traces = m.d_traces;
  a.fixmask = m.d_fixmask;
  a.fixval = m.d_fixval;
  a.sel = m.d_sel;
  a.psi = m.d_psi;
  a.eps = eps;
  a.box[0] = c->xmin[0]; a.box[1] = c->xmin[1]; a.box[2] = c->xmax[0]; a.box[3] = c->xmax[1];
  MCK(icx::launch_mdgjac(dm, c->phys, a, s));
  long long nbsr = (long long)dm.nnzb * dm.nb * dm.neq * dm.nb * dm.neq;
  icx::mdg_assemble_kernel<<<(unsigned)((m.nnz + 255) / 256), 256, 0, s>>>(m.nnz, m.d_src_ptr, m.d_src, nbsr, m.d_bsr,
                                                                         m.d_slots, d_csr_vals);
  MCK(cudaGetLastError());
  return ICX_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ LM solver
namespace icx {

// per element: minimum det J over the volume quadrature points < 0 -> *flag = 1
template <int G>
__global__ void min_det_kernel(DeviceMesh dm, int* flag) {
  constexpr int NG = (G + 1) * (G + 1);
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= dm.E * dm.nqv) return;
  int e = t / dm.nqv, q = t - e * dm.nqv;
  double J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int n = 0; n < NG; ++n) {
    int gn = dm.el_nodes[e * NG + n];
    double d0 = dm.tab_gvol[(q * NG + n) * 2], d1 = dm.tab_gvol[(q * NG + n) * 2 + 1];
    J[0][0] += d0 * dm.coord[2 * gn]; J[0][1] += d1 * dm.coord[2 * gn];
    J[1][0] += d0 * dm.coord[2 * gn + 1]; J[1][1] += d1 * dm.coord[2 * gn + 1];
  }
  if (J[0][0] * J[1][1] - J[0][1] * J[1][0] < 0.0) atomicExch(flag, 1);
}

// per element: minimum det J over the volume quadrature points (not clamped)
template <int G>
__global__ void elem_min_det_kernel(DeviceMesh dm, double* __restrict__ mins) {
  constexpr int NG = (G + 1) * (G + 1);
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= dm.E) return;
  double m = 1e100;
  for (int q = 0; q < dm.nqv; ++q) {
    double J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int n = 0; n < NG; ++n) {
      int gn = dm.el_nodes[e * NG + n];
      double d0 = dm.tab_gvol[(q * NG + n) * 2], d1 = dm.tab_gvol[(q * NG + n) * 2 + 1];
      J[0][0] += d0 * dm.coord[2 * gn]; J[0][1] += d1 * dm.coord[2 * gn];
      J[1][0] += d0 * dm.coord[2 * gn + 1]; J[1][1] += d1 * dm.coord[2 * gn + 1];
    }
    m = fmin(m, J[0][0] * J[1][1] - J[0][1] * J[1][0]);
  }
  mins[e] = m;
}

// A = J^T J on A's pattern: one warp per row i of A (column i of J); for each
// entry (r, J_ri) of column i the lanes add J_ri J_rc over row r of J into
// the positions of A's row i (binary search), rows r in ascending order
__global__ void jtj_kernel(long long n, const int* __restrict__ t_rowptr, const int* __restrict__ t_colidx,
                           const double* __restrict__ t_vals, const int* __restrict__ rowptr,
                           const int* __restrict__ colidx, const double* __restrict__ vals,
                           const int* __restrict__ a_rowptr, const int* __restrict__ a_colidx,
                           double* __restrict__ a_vals) {
  long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int a0 = a_rowptr[i], a1 = a_rowptr[i + 1];
  for (int k = a0 + lane; k < a1; k += 32) a_vals[k] = 0.0;
  __syncwarp();
  for (int t = t_rowptr[i]; t < t_rowptr[i + 1]; ++t) {
    const int r = t_colidx[t];
    const double v = t_vals[t];
    for (int q = rowptr[r] + lane; q < rowptr[r + 1]; q += 32) {
      const int c = colidx[q];
      int lo = a0, hi = a1 - 1;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a_colidx[mid] < c) lo = mid + 1;
        else hi = mid;
      }
      if (lo < a1 && a_colidx[lo] == c) a_vals[lo] += v * vals[q];
    }
    __syncwarp();
  }
}

// the column-norm scaled diagonal of the explicit subproblem:
// lambda_u |J_col| (PDE unknowns), lambda_b |J_col| (geometry) (corrigan_lm.hpp:429-451)
__global__ void a_diag_kernel(long long n, long long npde, double lu, double lb, const double* __restrict__ cn,
                              const int* __restrict__ a_diag, double* __restrict__ a_vals) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  a_vals[a_diag[i]] += (i < npde ? lu : lb) * cn[i];
}

// per element the stiffness K of the isoparametric continuous space (Lagrange
// order G, (G + 1)^2 Gauss-Legendre points, det J not clamped;
// DiffusionIntegrator, bilinear_integrators.hpp:11-49) and the pair values
// K[NG-1][il] K[NG-1][jl] lag + (il == jl ? lambda_el[e] : 0): the reference's
// K^T K loop assigns KTK[i][j] = K[k][i] K[k][j] for every k in turn, so the
// last basis function's row remains (corrigan_lm.hpp:463-469)
template <int G>
__global__ void lm_pair_kernel(DeviceMesh dm, const double* __restrict__ cg_tab, const int* __restrict__ pair_ptr,
                               const int* __restrict__ pair_ij, const double* __restrict__ lam_el, double lag,
                               double* __restrict__ pair_val) {
  constexpr int NG = (G + 1) * (G + 1), NQ = (G + 1) * (G + 1);
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= dm.E || pair_ptr[e] == pair_ptr[e + 1]) return;
  double xn[NG][2];
  for (int n = 0; n < NG; ++n) {
    int gn = dm.el_nodes[e * NG + n];
    xn[n][0] = dm.coord[2 * gn];
    xn[n][1] = dm.coord[2 * gn + 1];
  }
  double klast[NG];
  for (int j = 0; j < NG; ++j) klast[j] = 0.0;
  for (int q = 0; q < NQ; ++q) {
    const double* t = cg_tab + (size_t)q * NG * 2;
    double J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int n = 0; n < NG; ++n) {
      J[0][0] += t[2 * n] * xn[n][0]; J[0][1] += t[2 * n + 1] * xn[n][0];
      J[1][0] += t[2 * n] * xn[n][1]; J[1][1] += t[2 * n + 1] * xn[n][1];
    }
    double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    double dd = det == 0.0 ? 1.0 : det;  // the physical-gradient guard of the reference (finite_element.hpp:235-255)
    // grad phi_n = adj(J)^T-based reference gradient / det
    double gl0 = (t[2 * (NG - 1)] * J[1][1] - t[2 * (NG - 1) + 1] * J[1][0]) / dd;
    double gl1 = (-t[2 * (NG - 1)] * J[0][1] + t[2 * (NG - 1) + 1] * J[0][0]) / dd;
    double w = cg_tab[(size_t)NQ * NG * 2 + q];
    for (int j = 0; j < NG; ++j) {
      double g0 = (t[2 * j] * J[1][1] - t[2 * j + 1] * J[1][0]) / dd;
      double g1 = (-t[2 * j] * J[0][1] + t[2 * j + 1] * J[0][0]) / dd;
      klast[j] += (gl0 * g0 + gl1 * g1) * det * w;
    }
  }
  for (int pidx = pair_ptr[e]; pidx < pair_ptr[e + 1]; ++pidx) {
    int il = pair_ij[2 * pidx], jl = pair_ij[2 * pidx + 1];
    double v = klast[il] * klast[jl] * lag;
    if (il == jl && lam_el[e] > 0.0) v += lam_el[e];
    pair_val[pidx] = v;
  }
}

// A[pos] += the pair values of that position, in ascending pair order
__global__ void pair_gather_kernel(int npos, const int* __restrict__ upos, const int* __restrict__ upos_ptr,
                                   const int* __restrict__ upos_list, const double* __restrict__ pair_val,
                                   double* __restrict__ a_vals) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npos) return;
  double s = 0.0;
  for (int t = upos_ptr[k]; t < upos_ptr[k + 1]; ++t) s += pair_val[upos_list[t]];
  a_vals[upos[k]] += s;
}

// scalar ILU(0) of a CSR matrix in natural order, one level of rows per
// launch, one warp per row (IKJ): for each k < i of row i in ascending order,
// l_ik = a_ik / u_kk, then a_ij -= l_ik u_kj for j > k of row k present in row i
__global__ void csr_ilu_level_kernel(int nrows, const int* __restrict__ rows, const int* __restrict__ rowptr,
                                     const int* __restrict__ colidx, const int* __restrict__ diag,
                                     double* __restrict__ lu, int* err) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= nrows) return;
  const int i = rows[w];
  const int r0 = rowptr[i], r1 = rowptr[i + 1], di = diag[i];
  for (int p = r0; p < di; ++p) {
    const int k = colidx[p];
    const double ukk = lu[diag[k]];
    if (ukk == 0.0) {
      if (lane == 0) atomicExch(err, 1);
      return;
    }
    const double l = lu[p] / ukk;
    __syncwarp();
    if (lane == 0) lu[p] = l;
    for (int q = diag[k] + 1 + lane; q < rowptr[k + 1]; q += 32) {
      const int j = colidx[q];
      int lo = p + 1, hi = r1 - 1;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (colidx[mid] < j) lo = mid + 1;
        else hi = mid;
      }
      if (lo < r1 && colidx[lo] == j) lu[lo] -= l * lu[q];
    }
    __syncwarp();
  }
}

// one level of the ILU(0) triangular solves, one warp per row: forward
// y_i = b_i - sum_{k<i} l_ik y_k; backward x_i = (y_i - sum_{j>i} u_ij x_j) / u_ii
__global__ void csr_tri_level_kernel(int nrows, const int* __restrict__ rows, const int* __restrict__ rowptr,
                                     const int* __restrict__ colidx, const int* __restrict__ diag,
                                     const double* __restrict__ lu, const double* __restrict__ b,
                                     double* __restrict__ y, int upper) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= nrows) return;
  const int i = rows[w];
  const int d = diag[i];
  const int q0 = upper ? d + 1 : rowptr[i], q1 = upper ? rowptr[i + 1] : d;
  double s = 0.0;
  for (int q = q0 + lane; q < q1; q += 32) s += lu[q] * y[colidx[q]];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) y[i] = upper ? (b[i] - s) / lu[d] : b[i] - s;
}

// the same solves in one launch each, scheduled by data flow: warps claim
// rows in solve order (ascending for the forward solve, descending for the
// backward one) from a counter, wait for the rows their entries refer to
// (which were claimed earlier, by warps that are running, so every wait
// ends), and publish each result with a per-row flag set to this solve's
// epoch. A wait gives up after ~2^22 polls (or at once when an earlier wait
// has given up), sets *err and goes on, so the launch always ends.
__global__ void csr_tri_flow_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                    const int* __restrict__ diag, const double* __restrict__ lu,
                                    const double* __restrict__ b, double* y, int upper, unsigned* ready,
                                    unsigned epoch, unsigned* next, int* err) {
  const int lane = threadIdx.x & 31;
  volatile unsigned* vr = ready;
  volatile double* vy = y;
  while (true) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(next, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= (unsigned)n) break;
    const int i = upper ? n - 1 - (int)t : (int)t;
    const int d = diag[i];
    const int q0 = upper ? d + 1 : rowptr[i], q1 = upper ? rowptr[i + 1] : d;
    double s = 0.0;
    for (int q = q0 + lane; q < q1; q += 32) {
      const int k = colidx[q];
      unsigned spins = 0;
      while (vr[k] != epoch) {
        if (++spins > (1u << 22) || *(volatile int*)err) {
          atomicExch(err, 1);
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
      s += lu[q] * vy[k];
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) {
      vy[i] = upper ? (b[i] - s) / lu[d] : b[i] - s;
      __threadfence();
      vr[i] = epoch;
    }
    __syncwarp();
  }
}

}  // namespace icx

namespace {

icx_status ensure_lm(icx_ctx* c, int m) {
  icx_mdg_state& s = *c->mdg;
  long long n = s.ncol, nr = s.nrow;
  if (s.d_kV && s.kb.m >= m && s.kb.n == n) return ICX_OK;
  double** bufs[] = {&s.d_colnorm, &s.d_diag, &s.d_jtr, &s.d_p, &s.d_ustep, &s.d_x, &s.d_kw, &s.d_kz, &s.d_kr,
                     &s.d_colnorm2};
  for (double** b : bufs) {
    if (*b) cudaFree(*b);
    MCK(cudaMalloc((void**)b, sizeof(double) * n));
  }
  double** rbufs[] = {&s.d_tmp, &s.d_res, &s.d_rwork};
  for (double** b : rbufs) {
    if (*b) cudaFree(*b);
    MCK(cudaMalloc((void**)b, sizeof(double) * nr));
  }
  if (s.d_kV) cudaFree(s.d_kV);
  MCK(cudaMalloc((void**)&s.d_kV, sizeof(double) * (size_t)(m + 1) * n));
  if (s.d_kdh) cudaFree(s.d_kdh);
  MCK(cudaMalloc((void**)&s.d_kdh, sizeof(double) * 3 * (m + 2)));
  if (!s.lw.partial) MCK(cudaMalloc((void**)&s.lw.partial, sizeof(double) * 64 * icx::kMdotBlocks));
  s.kb.n = n;
  s.kb.m = m;
  s.kb.V = s.d_kV;
  s.kb.w = s.d_kw;
  s.kb.z = s.d_kz;
  s.kb.r = s.d_kr;
  s.kb.dh = s.d_kdh;
  s.kb.lw = &s.lw;
  return ICX_OK;
}

// the explicitly formed subproblem's pattern (A = J^T J over the unknowns
// [u; x], its diagonal, and the geometry pairs the Laplacian and the
// element-wise regularisation add to), its ILU(0) level schedules and the
// continuous-space tabulation; built once per selection (the pattern of J
// does not change when the nodes move)
icx_status build_lm_explicit(icx_ctx* c) {
  icx_mdg_state& m = *c->mdg;
  const icx::DeviceMesh& dm = c->dm;
  const long long n = m.ncol;
  const int g = c->geo_order, ng = (g + 1) * (g + 1);
  const long long N = (long long)dm.E * dm.nb * dm.neq;
  // geometry pairs per element: (il, jl, row, col) of the free coordinates of two selected nodes
  std::vector<int> pair_ptr(dm.E + 1, 0), pair_ij;
  std::vector<std::pair<long long, long long>> pair_rc;
  auto nfree = [&](int k) { return m.cols[k + 1] - m.cols[k]; };
  for (int e = 0; e < dm.E; ++e) {
    for (int il = 0; il < ng; ++il) {
      int ki = m.inv[c->el_nodes[(size_t)e * ng + il]];
      if (ki >= m.nsel) continue;
      for (int jl = 0; jl < ng; ++jl) {
        int kj = m.inv[c->el_nodes[(size_t)e * ng + jl]];
        if (kj >= m.nsel) continue;
        for (int iv = 0; iv < nfree(ki); ++iv)
          for (int jv = 0; jv < nfree(kj); ++jv) {
            pair_ij.push_back(il);
            pair_ij.push_back(jl);
            pair_rc.push_back({N + m.cols[ki] + iv, N + m.cols[kj] + jv});
          }
      }
    }
    pair_ptr[e + 1] = (int)pair_rc.size();
  }
  // A's pattern: row i = the union of the rows of J that column i touches, the diagonal and the pairs
  std::vector<std::vector<int>> extra(n);
  for (auto& rc : pair_rc) extra[rc.first].push_back((int)rc.second);
  std::vector<int> arow(n + 1, 0), acol, stamp(n, -1), cur;
  for (long long i = 0; i < n; ++i) {
    cur.clear();
    auto add = [&](int col) {
      if (stamp[col] != (int)i) {
        stamp[col] = (int)i;
        cur.push_back(col);
      }
    };
    add((int)i);
    for (int t = m.h_trowptr[i]; t < m.h_trowptr[i + 1]; ++t) {
      int r = m.h_tcolidx[t];
      for (int q = m.h_rowptr[r]; q < m.h_rowptr[r + 1]; ++q) add(m.h_colidx[q]);
    }
    for (int col : extra[i]) add(col);
    std::sort(cur.begin(), cur.end());
    acol.insert(acol.end(), cur.begin(), cur.end());
    arow[i + 1] = (int)acol.size();
  }
  m.a_nnz = (long long)acol.size();
  std::vector<int> adiag(n);
  auto find = [&](long long i, int col) {
    auto b = acol.begin() + arow[i], e = acol.begin() + arow[i + 1];
    return (int)(std::lower_bound(b, e, col) - acol.begin());
  };
  for (long long i = 0; i < n; ++i) adiag[i] = find(i, (int)i);
  // per touched position, its pairs in ascending order
  std::vector<std::pair<int, int>> pos_pair(pair_rc.size());
  for (size_t p = 0; p < pair_rc.size(); ++p) pos_pair[p] = {find(pair_rc[p].first, (int)pair_rc[p].second), (int)p};
  std::sort(pos_pair.begin(), pos_pair.end());
  std::vector<int> upos, uptr(1, 0), ulist;
  for (size_t t = 0; t < pos_pair.size(); ++t) {
    if (t == 0 || pos_pair[t].first != pos_pair[t - 1].first) {
      if (t) uptr.push_back((int)ulist.size());
      upos.push_back(pos_pair[t].first);
    }
    ulist.push_back(pos_pair[t].second);
  }
  uptr.push_back((int)ulist.size());
  if (pos_pair.empty()) uptr.assign(1, 0);
  m.npairs = (int)pair_rc.size();
  m.npos = (int)upos.size();
  // ILU(0) level schedules in natural order
  std::vector<int> lo(n, 0), upv(n, 0);
  int nlo = 0, nup = 0;
  for (long long i = 0; i < n; ++i) {
    int l = 0;
    for (int q = arow[i]; q < adiag[i]; ++q) l = std::max(l, lo[acol[q]] + 1);
    lo[i] = l;
    nlo = std::max(nlo, l + 1);
  }
  for (long long i = n - 1; i >= 0; --i) {
    int l = 0;
    for (int q = adiag[i] + 1; q < arow[i + 1]; ++q) l = std::max(l, upv[acol[q]] + 1);
    upv[i] = l;
    nup = std::max(nup, l + 1);
  }
  auto schedule = [&](const std::vector<int>& lv, int nl, std::vector<int>& off, std::vector<int>& rows) {
    off.assign(nl + 1, 0);
    for (int v : lv) ++off[v + 1];
    for (int l = 0; l < nl; ++l) off[l + 1] += off[l];
    rows.assign(n, 0);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (long long i = 0; i < n; ++i) rows[fill[lv[i]]++] = (int)i;
  };
  std::vector<int> lo_rows, up_rows;
  schedule(lo, nlo, m.lo_off, lo_rows);
  schedule(upv, nup, m.up_off, up_rows);
  // the continuous space's reference gradients at its (g + 1)^2 Gauss points, then the weights
  const int nq = g + 1;
  double qx[16], qw[16];
  icx::gauss_legendre_points(nq, qx, qw);
  std::vector<double> tab((size_t)nq * nq * ng * 2 + nq * nq);
  double N0[16], D0[16], N1[16], D1[16];
  for (int q0 = 0; q0 < nq; ++q0)
    for (int q1 = 0; q1 < nq; ++q1) {
      icx::lagrange_values_derivs(g, qx[q0], N0, D0);
      icx::lagrange_values_derivs(g, qx[q1], N1, D1);
      const int q = q0 * nq + q1;
      for (int a = 0; a <= g; ++a)
        for (int b = 0; b <= g; ++b) {
          const int k = a * (g + 1) + b;
          tab[((size_t)q * ng + k) * 2] = D0[a] * N1[b];
          tab[((size_t)q * ng + k) * 2 + 1] = N0[a] * D1[b];
        }
      tab[(size_t)nq * nq * ng * 2 + q] = qw[q0] * qw[q1];
    }
  MCK(up(&m.d_a_rowptr, arow));
  MCK(up(&m.d_a_colidx, acol));
  MCK(up(&m.d_a_diag, adiag));
  MCK(up(&m.d_lo_rows, lo_rows));
  MCK(up(&m.d_up_rows, up_rows));
  MCK(up(&m.d_pair_ptr, pair_ptr));
  MCK(up(&m.d_pair_ij, pair_ij.empty() ? std::vector<int>(2, 0) : pair_ij));
  MCK(up(&m.d_upos, upos.empty() ? std::vector<int>(1, 0) : upos));
  MCK(up(&m.d_upos_ptr, uptr));
  MCK(up(&m.d_upos_list, ulist.empty() ? std::vector<int>(1, 0) : ulist));
  MCK(up(&m.d_cg_tab, tab));
  for (double** b : {&m.d_a_vals, &m.d_a_lu}) {
    if (*b) cudaFree(*b);
    MCK(cudaMalloc((void**)b, sizeof(double) * std::max(m.a_nnz, 1LL)));
  }
  for (double** b : {&m.d_pair_val}) {
    if (*b) cudaFree(*b);
    MCK(cudaMalloc((void**)b, sizeof(double) * std::max(m.npairs, 1)));
  }
  for (double** b : {&m.d_lam_el, &m.d_detmin}) {
    if (*b) cudaFree(*b);
    MCK(cudaMalloc((void**)b, sizeof(double) * dm.E));
  }
  if (!m.d_pc_err) MCK(cudaMalloc((void**)&m.d_pc_err, sizeof(int)));
  if (m.d_tri_ready) cudaFree(m.d_tri_ready);
  MCK(cudaMalloc((void**)&m.d_tri_ready, sizeof(unsigned) * std::max(n, 1LL)));
  MCK(cudaMemset(m.d_tri_ready, 0, sizeof(unsigned) * std::max(n, 1LL)));
  m.tri_epoch = 0;
  if (!m.d_tri_next) MCK(cudaMalloc((void**)&m.d_tri_next, 2 * sizeof(unsigned)));
  if (!m.d_tri_err) MCK(cudaMalloc((void**)&m.d_tri_err, sizeof(int)));
  MCK(cudaMemset(m.d_tri_err, 0, sizeof(int)));
  m.a_built = true;
  return ICX_OK;
}

double corrigan_ls_lm(const std::function<double(double)>& f, double alpha_max, double alpha1, int kmax,
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

extern "C" {

icx_status icx_lm_default_options(icx_lm_options* o) {
  if (!o) return ICX_ERR_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->tau_abs = 1e-10;
  o->tau_rel = 0.0;
  o->kmax = 50;
  o->lambda_u = 1e-7;        // CorriganLM defaults (corrigan_lm.hpp:220-229)
  o->lambda_b = 1e-2;
  o->linesearch = 2;         // corrigan_linesearch defaults (nonlinear_solver_utils.hpp:236-257)
  o->ls_max_it = 20;
  o->ls_alpha_initial = 1.0;
  o->ls_alpha_max = 10.0;
  o->ls_alpha_min = 0.0;
  o->gmres_restart = 30;
  o->gmres_max_it = 10000;
  o->gmres_rtol = 1e-5;
  o->max_rejections = 20;
  o->explicit_subproblem = 0;  // CorriganLM's explicitly_form_subproblem default (corrigan_lm.hpp:286)
  o->lambda_lag = 1e-5;        // CorriganLM::lambda_lag (corrigan_lm.hpp:223)
  return ICX_OK;
}

icx_status icx_lm_solve(icx_ctx* c, double* d_u, double* x, const icx_lm_options* opt, icx_lm_report* rep) {
  if (!c || !c->mdg || !d_u || !x || !opt) return merr(c, ICX_ERR_INVALID, "MDG selection / arguments missing");
  if (opt->gmres_restart < 1 || opt->gmres_restart > 60) return merr(c, ICX_ERR_INVALID, "restart in 1..60");
  icx_mdg_state& s = *c->mdg;
  if (!s.d_rowptr) {
    icx_status st = build_mdg_pattern(c);
    if (st != ICX_OK) return st;
  }
  icx_status st = ensure_lm(c, opt->gmres_restart);
  if (st != ICX_OK) return st;
  cudaStream_t strm = 0;
  const icx::DeviceMesh& dm = c->dm;
  long long N = (long long)dm.E * dm.nb * dm.neq, n = s.ncol, nr = s.nrow, ngeo = s.ngeo;
  icx_lm_report local{};
  icx_lm_report* R = rep ? rep : &local;
  std::memset(R, 0, sizeof(*R));
  const double eps = std::sqrt(DBL_EPSILON);
  std::vector<double> xh(x, x + ngeo), xstep(ngeo), px(ngeo);
  st = icx_mdg_set_x(c, xh.data());
  if (st != ICX_OK) return st;
  auto form = [&]() -> icx_status {
    icx_status s2 = icx_form_jacobian_mdg_fd(c, d_u, s.d_res, s.d_res + N, s.d_vals, eps, strm);
    if (s2 != ICX_OK) return s2;
    icx::gather_kernel<<<(unsigned)((s.nnz + 255) / 256), 256, 0, strm>>>(s.nnz, s.d_t_perm, s.d_vals, s.d_tvals);
    return cudaGetLastError() == cudaSuccess ? ICX_OK : ICX_ERR_CUDA;
  };
  st = form();
  if (st != ICX_OK) return st;
  const bool explicit_sub = opt->explicit_subproblem != 0;
  if (explicit_sub && !s.a_built && (st = build_lm_explicit(c)) != ICX_OK) return st;
  double rk = icx::la_norm(s.lw, nr, s.d_res, s.d_kdh, strm);
  R->r0 = rk;
  R->residual_history[0] = rk;
  double tau = opt->tau_abs + opt->tau_rel * rk;
  double lu = opt->lambda_u, lb = opt->lambda_b, lu_min = lu;
  std::vector<double> lam_el(dm.E, 0.0), detmin(dm.E);  // element-wise regularisation (corrigan_lm.hpp:507-527)
  int k = 0, rejections = 0, hist = 0;
  bool converged = rk <= tau;
  int* d_flag = nullptr;
  MCK(cudaMalloc((void**)&d_flag, sizeof(int)));
  auto cleanup = [&]() { cudaFree(d_flag); };
  while (!converged && k < opt->kmax) {
    // J^T r and the regularisation from the column norms of J
    unsigned nb_n = (unsigned)((n * 32 + 255) / 256), nb_r = (unsigned)((nr * 32 + 255) / 256);
    icx::csr_rownorm_kernel<<<nb_n, 256, 0, strm>>>(n, s.d_t_rowptr, s.d_tvals, s.d_colnorm);
    icx::csr_spmv_kernel<<<nb_n, 256, 0, strm>>>(n, s.d_t_rowptr, s.d_t_colidx, s.d_tvals, s.d_res, s.d_jtr);
    icx::LinOp A, M;
    bool use_m = false;
    if (explicit_sub) {
      // A = J^T J + diag(lambda |J_col|) + lambda_lag |r| K^T K + lambda_el
      // (corrigan_lm.hpp:426-530), then its ILU(0) (the reference's PCILU)
      icx::jtj_kernel<<<nb_n, 256, 0, strm>>>(n, s.d_t_rowptr, s.d_t_colidx, s.d_tvals, s.d_rowptr, s.d_colidx,
                                               s.d_vals, s.d_a_rowptr, s.d_a_colidx, s.d_a_vals);
      icx::a_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, strm>>>(n, N, lu, lb, s.d_colnorm, s.d_a_diag,
                                                                         s.d_a_vals);
      if (s.npairs > 0) {
        MCK(cudaMemcpyAsync(s.d_lam_el, lam_el.data(), sizeof(double) * dm.E, cudaMemcpyHostToDevice, strm));
        const double lag = opt->lambda_lag * rk;
        if (dm.G == 1)
          icx::lm_pair_kernel<1><<<(dm.E + 127) / 128, 128, 0, strm>>>(dm, s.d_cg_tab, s.d_pair_ptr, s.d_pair_ij,
                                                                      s.d_lam_el, lag, s.d_pair_val);
        else
          icx::lm_pair_kernel<2><<<(dm.E + 127) / 128, 128, 0, strm>>>(dm, s.d_cg_tab, s.d_pair_ptr, s.d_pair_ij,
                                                                      s.d_lam_el, lag, s.d_pair_val);
        icx::pair_gather_kernel<<<(s.npos + 255) / 256, 256, 0, strm>>>(s.npos, s.d_upos, s.d_upos_ptr,
                                                                        s.d_upos_list, s.d_pair_val, s.d_a_vals);
      }
      MCK(cudaMemcpyAsync(s.d_a_lu, s.d_a_vals, sizeof(double) * s.a_nnz, cudaMemcpyDeviceToDevice, strm));
      MCK(cudaMemsetAsync(s.d_pc_err, 0, sizeof(int), strm));
      for (size_t l = 0; l + 1 < s.lo_off.size(); ++l) {
        const int cnt = s.lo_off[l + 1] - s.lo_off[l];
        icx::csr_ilu_level_kernel<<<(cnt * 32 + 255) / 256, 256, 0, strm>>>(
            cnt, s.d_lo_rows + s.lo_off[l], s.d_a_rowptr, s.d_a_colidx, s.d_a_diag, s.d_a_lu, s.d_pc_err);
      }
      MCK(cudaGetLastError());
      int perr = 0;
      MCK(cudaMemcpyAsync(&perr, s.d_pc_err, sizeof(int), cudaMemcpyDeviceToHost, strm));
      MCK(cudaStreamSynchronize(strm));
      if (perr) { cleanup(); return merr(c, ICX_ERR_NONFINITE, "LM subproblem ILU(0): zero pivot"); }
      A = [&](const double* xin, double* yout, cudaStream_t st) {
        icx::csr_spmv_kernel<<<nb_n, 256, 0, st>>>(n, s.d_a_rowptr, s.d_a_colidx, s.d_a_vals, xin, yout);
        return cudaGetLastError();
      };
      // the two triangular solves, one data-flow launch each (the level
      // schedule would take one launch per level, ~2 x 760 at 64 x 64)
      M = [&](const double* xin, double* yout, cudaStream_t st) {
        const unsigned e_l = ++s.tri_epoch, e_u = ++s.tri_epoch;
        const int nn = (int)n;
        const unsigned grid = (unsigned)std::min<long long>((n + 7) / 8, 148LL * 8);
        cudaError_t e = cudaMemsetAsync(s.d_tri_next, 0, 2 * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
        icx::csr_tri_flow_kernel<<<grid, 256, 0, st>>>(nn, s.d_a_rowptr, s.d_a_colidx, s.d_a_diag, s.d_a_lu, xin,
                                                       s.d_colnorm2, 0, s.d_tri_ready, e_l, s.d_tri_next, s.d_tri_err);
        icx::csr_tri_flow_kernel<<<grid, 256, 0, st>>>(nn, s.d_a_rowptr, s.d_a_colidx, s.d_a_diag, s.d_a_lu,
                                                       s.d_colnorm2, yout, 1, s.d_tri_ready, e_u, s.d_tri_next + 1,
                                                       s.d_tri_err);
        return cudaGetLastError();
      };
      use_m = true;
    } else {
      icx::lm_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, strm>>>(n, N, lu, lb, s.d_colnorm, s.d_diag);
      A = [&](const double* xin, double* yout, cudaStream_t st) {
        icx::csr_spmv_kernel<<<nb_r, 256, 0, st>>>(nr, s.d_rowptr, s.d_colidx, s.d_vals, xin, s.d_tmp);
        icx::csr_spmv_kernel<<<nb_n, 256, 0, st>>>(n, s.d_t_rowptr, s.d_t_colidx, s.d_tvals, s.d_tmp, yout);
        icx::diag_axpy_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, s.d_diag, xin, yout);
        return cudaGetLastError();
      };
    }
    int its = 0;
    double rr = 0.0;
    st = icx::gmres_op(s.kb, A, use_m ? &M : nullptr, opt->gmres_max_it, opt->gmres_rtol, s.d_jtr, s.d_p, &its, &rr,
                       strm, &c->err);
    if (st != ICX_OK) { cleanup(); return st; }
    if (use_m) {
      int terr = 0;
      MCK(cudaMemcpyAsync(&terr, s.d_tri_err, sizeof(int), cudaMemcpyDeviceToHost, strm));
      MCK(cudaStreamSynchronize(strm));
      if (terr) {
        cudaMemset(s.d_tri_err, 0, sizeof(int));
        cudaMemset(s.d_tri_ready, 0, sizeof(unsigned) * n);
        s.tri_epoch = 0;
        cleanup();
        return merr(c, ICX_ERR_CUDA, "LM subproblem ILU(0) apply: a dependency wait timed out");
      }
    }
    R->linear_iterations_total += its;
    R->linear_relres_max = std::max(R->linear_relres_max, rr);
    MCK(cudaMemcpy(px.data(), s.d_p + N, sizeof(double) * ngeo, cudaMemcpyDeviceToHost));
    if (opt->step_only) {
      // the first subproblem's solution in place of the unknowns
      MCK(cudaMemcpyAsync(d_u, s.d_p, sizeof(double) * N, cudaMemcpyDeviceToDevice, strm));
      MCK(cudaStreamSynchronize(strm));
      std::memcpy(x, px.data(), sizeof(double) * ngeo);
      cleanup();
      return icx_mdg_set_x(c, xh.data());  // the mesh stays at the input nodes
    }
    double alpha = 1.0;
    bool accept = true;
    if (opt->linesearch == 2) {
      double rnorm_old = rk, rnorm_step = 0.0;
      std::function<double(double)> phi = [&](double a) -> double {
        icx::la_xpay(N, d_u, -a, s.d_p, s.d_ustep, strm);
        for (long long i = 0; i < ngeo; ++i) xstep[i] = xh[i] - a * px[i];
        icx_status s3 = icx_mdg_set_x(c, xstep.data());
        if (s3 != ICX_OK) return NAN;
        icx_form_residual(c, s.d_ustep, s.d_rwork, strm);
        icx_form_mdg_residual(c, s.d_ustep, s.d_rwork + N, strm);
        double v = icx::la_norm(s.lw, N, s.d_rwork, s.d_kdh, strm) +
                   icx::la_norm(s.lw, nr - N, s.d_rwork + N, s.d_kdh, strm);
        rnorm_step = v;
        return v;
      };
      alpha = corrigan_ls_lm(phi, opt->ls_alpha_max, opt->ls_alpha_initial, opt->ls_max_it, opt->ls_alpha_min);
      // element inversion check on the last line-search mesh, with the
      // element-wise regularisation updates (corrigan_lm.hpp:625-666)
      bool inverted = false;
      if (explicit_sub) {
        if (dm.G == 1) icx::elem_min_det_kernel<1><<<(dm.E + 127) / 128, 128, 0, strm>>>(dm, s.d_detmin);
        else icx::elem_min_det_kernel<2><<<(dm.E + 127) / 128, 128, 0, strm>>>(dm, s.d_detmin);
        MCK(cudaMemcpy(detmin.data(), s.d_detmin, sizeof(double) * dm.E, cudaMemcpyDeviceToHost));
        for (int e = 0; e < dm.E; ++e)
          if (detmin[e] < 0.0) {
            inverted = true;
            lam_el[e] = lam_el[e] == 0.0 ? lb : lam_el[e] * std::max(1.5, std::fabs(detmin[e]));
          }
      } else {
        cudaMemset(d_flag, 0, sizeof(int));
        if (dm.G == 1) icx::min_det_kernel<1><<<(dm.E * dm.nqv + 255) / 256, 256, 0, strm>>>(dm, d_flag);
        else icx::min_det_kernel<2><<<(dm.E * dm.nqv + 255) / 256, 256, 0, strm>>>(dm, d_flag);
        int fl = 0;
        MCK(cudaMemcpy(&fl, d_flag, sizeof(int), cudaMemcpyDeviceToHost));
        inverted = fl != 0;
      }
      accept = !inverted && rnorm_step < 10 * rnorm_old;
      if (accept) {
        lu = std::max(lu_min, 0.55 * lu);
        lb = std::max(rnorm_step, 0.55 * lb);
        for (double& l : lam_el)
          if (l > 0.0) l /= 1.5;
      } else {
        lu *= 1.8;
        lb *= 1.8;
      }
    }
    if (accept) {
      icx::la_axpby(N, -alpha, s.d_p, 1.0, d_u, strm);
      for (long long i = 0; i < ngeo; ++i) xh[i] -= alpha * px[i];
      rejections = 0;
    } else {
      ++rejections;
      ++R->rejections;
    }
    st = icx_mdg_set_x(c, xh.data());
    if (st != ICX_OK) { cleanup(); return st; }
    if (!accept) {
      if (rejections > opt->max_rejections) { cleanup(); return merr(c, ICX_ERR_NOT_CONVERGED, "too many rejected LM steps"); }
      continue;  // retry with the larger regularisation
    }
    st = form();
    if (st != ICX_OK) { cleanup(); return st; }
    rk = icx::la_norm(s.lw, nr, s.d_res, s.d_kdh, strm);
    ++k;
    if (++hist < 64) {
      R->residual_history[hist] = rk;
      R->alpha_history[hist - 1] = alpha;
    }
    if (opt->verbosity > 0)
      std::printf("lm %d: |r| = %.6e alpha = %.4f gmres its = %d relres = %.3e\n", k, rk, alpha, its, rr);
    if (!std::isfinite(rk)) { cleanup(); return merr(c, ICX_ERR_NONFINITE, "non-finite residual"); }
    converged = rk <= tau;
  }
  cleanup();
  std::memcpy(x, xh.data(), sizeof(double) * ngeo);
  R->iterations = k;
  R->converged = converged;
  R->r_final = rk;
  return converged ? ICX_OK : ICX_ERR_NOT_CONVERGED;
}

}  // extern "C"
