// Host side of the C ABI: mesh construction in the reference's ordering,
// finite element space tabulations, boundary/source data through the user's
// callbacks, device table upload and the residual entry point.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "icx_internal.h"

using icx::DeviceMesh;

namespace {

icx_status fail(icx_ctx* c, icx_status st, const char* msg) {
  if (c) c->err = msg;
  return st;
}

icx_status cuda_fail(icx_ctx* c, cudaError_t e, const char* where) {
  if (c) c->err = std::string(where) + ": " + cudaGetErrorString(e);
  return ICX_ERR_CUDA;
}

// ---------------------------------------------------------------- 1D bases
// Lagrange polynomials through pn+1 equispaced nodes of [-1, 1] (node j
// accumulated as x_{j-1} + 2/pn, lagrange_1d.hpp:30-42), evaluated in
// barycentric form with the node nearest to x factored out (lagrange_1d.hpp:78-118).
// 1D basis of order pn on [-1, 1]: Lagrange polynomials through equispaced
// nodes (kind ICX_BASIS_LAGRANGE), or the Legendre polynomials P_0..P_pn
// (kind ICX_BASIS_LEGENDRE, unnormalised, P_k(1) = 1)
struct Lagrange1D {
  int pn;
  int kind = ICX_BASIS_LAGRANGE;
  double xi[16], wj[16];
  Lagrange1D(int n, int k) : Lagrange1D(n) { kind = k; }
  explicit Lagrange1D(int n) : pn(n) {
    xi[0] = -1.0;
    double dx = 2.0 / pn;
    for (int j = 1; j <= pn; ++j) xi[j] = xi[j - 1] + dx;
    for (int j = 0; j <= pn; ++j) {
      double w = 1.0;
      for (int k = 0; k <= pn; ++k)
        if (k != j) w *= (xi[j] - xi[k]);
      wj[j] = 1.0 / w;
    }
  }
  // P_0..P_pn with first and second derivatives by the three-term recurrence
  // (k+1) P_{k+1} = (2k+1) x P_k - k P_{k-1}, differentiated once and twice
  void legendre(double x, double* N, double* dN, double* d2N) const {
    N[0] = 1.0;
    dN[0] = 0.0;
    d2N[0] = 0.0;
    if (pn >= 1) {
      N[1] = x;
      dN[1] = 1.0;
      d2N[1] = 0.0;
    }
    for (int k = 1; k < pn; ++k) {
      const double a = (2.0 * k + 1.0) / (k + 1.0), b = (double)k / (k + 1.0);
      N[k + 1] = a * x * N[k] - b * N[k - 1];
      dN[k + 1] = a * (N[k] + x * dN[k]) - b * dN[k - 1];
      d2N[k + 1] = a * (2.0 * dN[k] + x * d2N[k]) - b * d2N[k - 1];
    }
  }
  void eval(double x, double* N, double* dN, double* d2N) const {
    if (kind == ICX_BASIS_LEGENDRE) {
      legendre(x, N, dN, d2N);
      return;
    }
    if (pn == 1) {
      N[0] = 0.5 * (1 - x);
      N[1] = 1.0 - N[0];
      dN[0] = -0.5;
      dN[1] = 0.5;
      d2N[0] = d2N[1] = 0.0;
      return;
    }
    double lskip = 1.0;
    int k;
    for (k = 0; k < pn; ++k) {
      if (x >= (xi[k] + xi[k + 1]) / 2) lskip *= (x - xi[k]);
      else break;
    }
    for (int i = k + 1; i <= pn; ++i) lskip *= (x - xi[i]);
    double lprod = lskip * (x - xi[k]);
    double s = 0.0;
    for (int j = 0; j <= pn; ++j) {
      if (j == k) continue;
      double inv = 1.0 / (x - xi[j]);
      s += inv;
      N[j] = lprod * inv * wj[j];
    }
    N[k] = lskip * wj[k];
    double lprime = lprod * s + lskip;
    for (int j = 0; j <= pn; ++j)
      dN[j] = (j == k) ? s * N[k] : (lprime * wj[j] - N[j]) / (x - xi[j]);
    // second derivative of the product form: 2 sum_{a<b} prod_{m != j,a,b} (x - x_m) / prod_{m!=j}(x_j - x_m)
    for (int j = 0; j <= pn; ++j) {
      double nodes_j = -1.0 + 2.0 * j / pn;
      double denom = 1.0;
      for (int m = 0; m <= pn; ++m)
        if (m != j) denom *= (nodes_j - (-1.0 + 2.0 * m / pn));
      double sum = 0.0;
      for (int a = 0; a <= pn; ++a) {
        if (a == j) continue;
        for (int b = a + 1; b <= pn; ++b) {
          if (b == j) continue;
          double p = 1.0;
          for (int m = 0; m <= pn; ++m)
            if (m != j && m != a && m != b) p *= (x - (-1.0 + 2.0 * m / pn));
          sum += p;
        }
      }
      d2N[j] = 2.0 * sum / denom;
    }
  }
};

// Gauss-Legendre points in the order (+x1, -x1, +x2, -x2, ..., 0) with
// Newton iteration on P_n from cos(pi (i - 1/4) / (n + 1/2)) (quadrules_1d.hpp:33-76)
void gauss_legendre(int n, double* x, double* w) {
  auto leg = [n](double t, double& P, double& dP) {
    double pkm1 = 1.0, pk = t, dkm1 = 0.0, dk = 1.0;
    for (int k = 1; k < n; ++k) {
      double pkp1 = ((2 * k + 1) * t * pk - k * pkm1) / (k + 1);
      double dkp1 = dkm1 + (2 * k + 1) * pk;
      pkm1 = pk; pk = pkp1; dkm1 = dk; dk = dkp1;
    }
    P = pk; dP = dk;
  };
  double wc = 2.0;
  for (int i = 1; i <= n / 2; ++i) {
    double t = std::cos(M_PI * (i - 0.25) / (n + 0.5));
    double P, dP;
    for (int it = 0; it < 50; ++it) {
      leg(t, P, dP);
      double d = P / dP;
      t -= d;
      if (std::fabs(d) < 1e-16) break;
    }
    leg(t, P, dP);
    double wt = 2.0 / ((1 - t * t) * dP * dP);
    wc -= 2 * wt;
    x[2 * (i - 1)] = t; w[2 * (i - 1)] = wt;
    x[2 * (i - 1) + 1] = -t; w[2 * (i - 1) + 1] = wt;
  }
  if (n % 2) { x[n - 1] = 0.0; w[n - 1] = wc; }
}

// reference coordinates of trace coordinate s on local face fn
// (HypercubeTraceTransformation::transform, HypercubeTransformations.hpp:1215-1236)
void face_ref(int fn, double s, double xi[2]) {
  switch (fn) {
    case 0: xi[0] = -1.0; xi[1] = -s; break;
    case 1: xi[0] = s; xi[1] = -1.0; break;
    case 2: xi[0] = 1.0; xi[1] = s; break;
    default: xi[0] = -s; xi[1] = 1.0; break;
  }
}

// tensor-product basis (dim 0 slowest) at xi: [nb][6] = phi, d0, d1, h00, h01, h11
void tp_tab(const Lagrange1D& l, const double xi[2], double* out) {
  int n = l.pn + 1;
  double N0[16], N1[16], a0[16], a1[16], s0[16], s1[16];
  l.eval(xi[0], N0, a0, s0);
  l.eval(xi[1], N1, a1, s1);
  for (int i0 = 0; i0 < n; ++i0)
    for (int i1 = 0; i1 < n; ++i1) {
      double* o = out + (i0 * n + i1) * 6;
      o[0] = N0[i0] * N1[i1];
      o[1] = a0[i0] * N1[i1];
      o[2] = N0[i0] * a1[i1];
      o[3] = s0[i0] * N1[i1];
      o[4] = a0[i0] * a1[i1];
      o[5] = N0[i0] * s1[i1];
    }
}

template <class T>
cudaError_t upload(T** dptr, const std::vector<T>& h) {
  if (*dptr) { cudaFree(*dptr); *dptr = nullptr; }
  if (h.empty()) return cudaSuccess;
  cudaError_t e = cudaMalloc((void**)dptr, sizeof(T) * h.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dptr, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
}

void free_dev(DeviceMesh& dm) {
  void* ptrs[] = {dm.coord, dm.el_nodes, dm.face_info, dm.el_face, dm.el_side, dm.el_fso, dm.el_par, dm.vgeo, dm.fgeo,
                  dm.tab_vol, dm.tab_face, dm.tab_1d, dm.tab_fphi, dm.tab_f1d, dm.tab_gvol, dm.tab_gface, dm.tab_gcen, dm.qw_face,
                  dm.bvals, dm.src, dm.face_flux, dm.face_grad, dm.bsr_rowptr, dm.bsr_colidx,
                  dm.bsr_diag, dm.face_blk};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  dm = DeviceMesh{};
}

int n_nodes(const icx_ctx* c) { return (int)(c->coord.size() / 2); }

// physical point of element e at reference xi via its geometry nodes
void el_point(const icx_ctx* c, const Lagrange1D& lg, int e, const double xi[2], double x[2]) {
  int ng = (c->geo_order + 1) * (c->geo_order + 1);
  std::vector<double> tab(ng * 6);
  tp_tab(lg, xi, tab.data());
  x[0] = x[1] = 0.0;
  for (int n = 0; n < ng; ++n) {
    int gn = c->el_nodes[e * ng + n];
    x[0] += tab[n * 6] * c->coord[2 * gn];
    x[1] += tab[n * 6] * c->coord[2 * gn + 1];
  }
}

// a batch takes its parts' boundary and source tables (already evaluated
// through their callbacks) in the batch's face and element order
icx_status batch_tables(icx_ctx* c) {
  DeviceMesh& dm = c->dm;
  const int neq = dm.neq;
  cudaError_t e = cudaSuccess;
  if (dm.bvals) { cudaFree(dm.bvals); dm.bvals = nullptr; }
  if (dm.src) { cudaFree(dm.src); dm.src = nullptr; }
  e = cudaMalloc((void**)&dm.bvals, sizeof(double) * (size_t)std::max(dm.Fb, 1) * dm.nqf * neq);
  if (e != cudaSuccess) return cuda_fail(c, e, "allocate boundary data");
  bool any_src = false;
  for (icx_ctx* pc : c->parts) any_src = any_src || pc->dm.src != nullptr;
  if (any_src) {
    e = cudaMalloc((void**)&dm.src, sizeof(double) * (size_t)dm.E * dm.nqv * neq);
    if (e == cudaSuccess) e = cudaMemset(dm.src, 0, sizeof(double) * (size_t)dm.E * dm.nqv * neq);
    if (e != cudaSuccess) return cuda_fail(c, e, "allocate source");
  }
  size_t boff = 0, eoff = 0;
  for (icx_ctx* pc : c->parts) {
    const DeviceMesh& pm = pc->dm;
    if (pm.Fb > 0 && (e = cudaMemcpy(dm.bvals + boff * dm.nqf * neq, pm.bvals,
                                     sizeof(double) * (size_t)pm.Fb * dm.nqf * neq, cudaMemcpyDeviceToDevice)) !=
                         cudaSuccess)
      return cuda_fail(c, e, "copy boundary data");
    if (pm.src && (e = cudaMemcpy(dm.src + eoff * dm.nqv * neq, pm.src, sizeof(double) * (size_t)pm.E * dm.nqv * neq,
                                  cudaMemcpyDeviceToDevice)) != cudaSuccess)
      return cuda_fail(c, e, "copy source");
    boff += pm.Fb;
    eoff += pm.E;
  }
  if ((e = upload(&dm.el_par, c->el_par)) != cudaSuccess) return cuda_fail(c, e, "upload element parameters");
  if ((e = upload(&dm.coord, c->coord)) != cudaSuccess) return cuda_fail(c, e, "upload coordinates");
  e = icx::launch_geometry(dm, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(c, e, "geometry kernels");
  return ICX_OK;
}

// boundary data and source through the callbacks, then geometry kernels
icx_status tabulate_and_geometry(icx_ctx* c) {
  if (!c->parts.empty()) return batch_tables(c);
  DeviceMesh& dm = c->dm;
  Lagrange1D lg(c->geo_order);
  double qx[16], qw[16];
  gauss_legendre(dm.nq1, qx, qw);
  int neq = dm.neq;
  // boundary values at boundary face points
  std::vector<double> bv((size_t)std::max(dm.Fb, 1) * dm.nqf * neq, 0.0);
  for (int f = c->n_interior; f < dm.F; ++f) {
    const int* F = &c->faces[7 * f];
    int bidx = f - c->n_interior;
    int bct = F[5], flag = F[6];
    icx_point_fn fn = nullptr;
    void* user = nullptr;
    if (bct == ICX_BC_DIRICHLET) {
      if (flag < 0 || flag >= (int)c->dirichlet_fn.size() || !c->dirichlet_fn[flag])
        return fail(c, ICX_ERR_INVALID, "missing Dirichlet callback for a boundary flag");
      fn = c->dirichlet_fn[flag]; user = c->dirichlet_user[flag];
    } else if (bct == ICX_BC_NEUMANN) {
      if (flag < 0 || flag >= (int)c->neumann_fn.size() || !c->neumann_fn[flag])
        return fail(c, ICX_ERR_INVALID, "missing Neumann callback for a boundary flag");
      fn = c->neumann_fn[flag]; user = c->neumann_user[flag];
    }
    if (c->phys.pde == ICX_PDE_NAVIER_STOKES &&
        (bct == ICX_BC_NO_SLIP_ISOTHERMAL || (bct == ICX_BC_WALL_GENERAL && c->phys.ns_viscous_wall))) {
      // the wall temperature of the face's bcflag (Physics::isothermal_temperatures[bcflag])
      if (flag < 0 || flag >= (int)c->wall_T.size())
        return fail(c, ICX_ERR_INVALID, "no wall temperature for an isothermal wall's boundary flag "
                                        "(icx_disc_ns_boundary)");
      for (int q = 0; q < dm.nqf; ++q) bv[((size_t)bidx * dm.nqf + q) * neq] = c->wall_T[flag];
      continue;
    }
    if (!fn) continue;
    for (int q = 0; q < dm.nqf; ++q) {
      double xi[2], x[2];
      face_ref(F[2], qx[q], xi);
      el_point(c, lg, F[0], xi, x);
      fn(x, &bv[((size_t)bidx * dm.nqf + q) * neq], user);
    }
  }
  cudaError_t e = upload(&dm.bvals, bv);
  if (e != cudaSuccess) return cuda_fail(c, e, "upload boundary data");
  c->phys.st_connected = 0;  // a past-slab connection holds for the mesh it was made on
  if (c->source_fn) {
    std::vector<double> sv((size_t)dm.E * dm.nqv * neq, 0.0);
    for (int el = 0; el < dm.E; ++el)
      for (int q0 = 0; q0 < dm.nq1; ++q0)
        for (int q1 = 0; q1 < dm.nq1; ++q1) {
          double xi[2] = {qx[q0], qx[q1]}, x[2];
          el_point(c, lg, el, xi, x);
          c->source_fn(x, &sv[((size_t)el * dm.nqv + q0 * dm.nq1 + q1) * neq], c->source_user);
        }
    e = upload(&dm.src, sv);
    if (e != cudaSuccess) return cuda_fail(c, e, "upload source");
  }
  e = upload(&dm.coord, c->coord);
  if (e != cudaSuccess) return cuda_fail(c, e, "upload coordinates");
  e = icx::launch_geometry(dm, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(c, e, "geometry kernels");
  return ICX_OK;
}

}  // namespace

namespace icx {
icx_status refresh_geometry(icx_ctx* c) { return tabulate_and_geometry(c); }
}  // namespace icx

extern "C" icx_status icx_spacetime_connect(icx_ctx* c, const icx_ctx* past, const double* d_u_past) {
  if (!c || !past || !d_u_past || !c->ready || !past->ready) return fail(c, ICX_ERR_INVALID, "contexts not set up");
  if (!c->phys.spacetime || !past->phys.spacetime || !c->parts.empty() || !past->parts.empty())
    return fail(c, ICX_ERR_INVALID, "both contexts must be single spacetime Burgers slabs");
  const icx::DeviceMesh& dm = c->dm;
  const int neq = dm.neq, nqf = dm.nqf;
  cudaSetDevice(past->device);
  const size_t np = (size_t)past->dm.E * past->dm.nb * past->dm.neq;
  std::vector<double> up(np);
  if (cudaMemcpy(up.data(), d_u_past, sizeof(double) * np, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(c, ICX_ERR_CUDA, "copy of the past state");
  // elements of the past slab on its SPACETIME_FUTURE faces (its top)
  std::vector<int> tops;
  for (size_t f = past->n_interior; f < past->faces.size() / 7; ++f)
    if (past->faces[7 * f + 5] == ICX_BC_SPACETIME_FUTURE) tops.push_back(past->faces[7 * f]);
  if (tops.empty()) return fail(c, ICX_ERR_INVALID, "the past slab has no SPACETIME_FUTURE faces");
  Lagrange1D lg(c->geo_order), lgp(past->geo_order), lbp(past->p, past->basis);
  double qx[16], qw[16];
  gauss_legendre(nqf, qx, qw);
  const int nbp1 = past->p + 1;
  cudaSetDevice(c->device);
  int n_faces = 0;
  for (size_t f = c->n_interior; f < c->faces.size() / 7; ++f) {
    const int* F = &c->faces[7 * f];
    if (F[5] != ICX_BC_SPACETIME_PAST) continue;
    ++n_faces;
    const int bidx = (int)f - c->n_interior;
    // the interface must lie at constant t: the face's end points share t
    double xa[2], xb[2], xi[2];
    face_ref(F[2], -1.0, xi);
    el_point(c, lg, F[0], xi, xa);
    face_ref(F[2], 1.0, xi);
    el_point(c, lg, F[0], xi, xb);
    if (std::fabs(xa[1] - xb[1]) > 1e-12 * (1.0 + std::fabs(xa[1])))
      return fail(c, ICX_ERR_UNSUPPORTED, "SPACETIME_PAST face not at constant t");
    std::vector<double> vals((size_t)nqf * neq);
    for (int q = 0; q < nqf; ++q) {
      double x[2];
      face_ref(F[2], qx[q], xi);
      el_point(c, lg, F[0], xi, x);
      // the past element whose top edge x(s, +1) passes through x: bisection on s
      bool found = false;
      for (int e : tops) {
        double s0 = -1.0, s1 = 1.0, p0[2], p1[2], r0[2] = {-1.0, 1.0}, r1[2] = {1.0, 1.0};
        el_point(past, lgp, e, r0, p0);
        el_point(past, lgp, e, r1, p1);
        const double tol = 1e-12 * (1.0 + std::fabs(x[0]));
        if ((x[0] - p0[0]) * (x[0] - p1[0]) > 0.0 && std::fabs(x[0] - p0[0]) > tol && std::fabs(x[0] - p1[0]) > tol)
          continue;
        if (std::fabs(p0[1] - x[1]) > 1e-9 * (1.0 + std::fabs(x[1])))
          return fail(c, ICX_ERR_INVALID, "the slabs do not meet: past top and current bottom differ in t");
        const double dir = p1[0] > p0[0] ? 1.0 : -1.0;
        for (int it = 0; it < 200 && s1 - s0 > 1e-15; ++it) {
          double sm = 0.5 * (s0 + s1), rm[2] = {sm, 1.0}, pm[2];
          el_point(past, lgp, e, rm, pm);
          if (dir * (pm[0] - x[0]) < 0.0) s0 = sm;
          else s1 = sm;
        }
        const double s = 0.5 * (s0 + s1);
        double N0[16], N1[16], dN[16], d2N[16];
        lbp.eval(s, N0, dN, d2N);
        lbp.eval(1.0, N1, dN, d2N);
        for (int eq = 0; eq < neq; ++eq) {
          double v = 0.0;
          for (int i0 = 0; i0 < nbp1; ++i0)
            for (int i1 = 0; i1 < nbp1; ++i1)
              v += up[((size_t)e * nbp1 * nbp1 + i0 * nbp1 + i1) * neq + eq] * N0[i0] * N1[i1];
          vals[(size_t)q * neq + eq] = v;
        }
        found = true;
        break;
      }
      if (!found) return fail(c, ICX_ERR_INVALID, "a SPACETIME_PAST point lies outside the past slab's top");
    }
    if (cudaMemcpy(dm.bvals + (size_t)bidx * nqf * neq, vals.data(), sizeof(double) * vals.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(c, ICX_ERR_CUDA, "upload of the past trace");
  }
  if (!n_faces) return fail(c, ICX_ERR_INVALID, "the context has no SPACETIME_PAST faces");
  c->phys.st_connected = 1;
  return ICX_OK;
}

namespace icx {
void lagrange_values(int pn, double x, double* N) {
  Lagrange1D l(pn);
  double dN[16], d2N[16];
  l.eval(x, N, dN, d2N);
}
void basis_values(int kind, int pn, double x, double* N) {
  Lagrange1D l(pn, kind);
  double dN[16], d2N[16];
  l.eval(x, N, dN, d2N);
}
void lagrange_values_derivs(int pn, double x, double* N, double* dN) {
  Lagrange1D l(pn);
  double d2N[16];
  l.eval(x, N, dN, d2N);
}
void gauss_legendre_points(int n, double* x, double* w) { gauss_legendre(n, x, w); }
void element_point(const icx_ctx* c, int e, const double xi[2], double x[2]) {
  Lagrange1D lg(c->geo_order);
  el_point(c, lg, e, xi, x);
}
}  // namespace icx

extern "C" {

icx_status icx_create(icx_ctx** out, int device) {
  if (!out) return ICX_ERR_INVALID;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return ICX_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return ICX_ERR_INVALID;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return ICX_ERR_CUDA;
  icx_ctx* c = new icx_ctx();
  c->device = device;
  *out = c;
  return ICX_OK;
}

void icx_destroy(icx_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  icx::free_solver_work(c);
  icx::free_mdg(c);
  icx::free_explicit(c);
  icx::free_lpc_work(c);
  icx::free_host_pipe(c);
  free_dev(c->dm);
  for (void* p : c->scratch)
    if (p) cudaFree(p);
  delete c;
}

const char* icx_last_error(const icx_ctx* c) { return c ? c->err.c_str() : "null context"; }

icx_status icx_mesh_uniform(icx_ctx* c, int ndim, const int* nelem, const double* xmin, const double* xmax,
                            int geo_order, const int* bctypes, const int* bcflags) {
  if (!c || !nelem || !xmin || !xmax || !bctypes || !bcflags) return fail(c, ICX_ERR_INVALID, "null argument");
  if (ndim != 2) return fail(c, ICX_ERR_UNSUPPORTED, "only 2D meshes are implemented");
  if (geo_order < 1 || geo_order > icx::MAX_G) return fail(c, ICX_ERR_UNSUPPORTED, "geometry order must be 1 or 2");
  if (nelem[0] < 1 || nelem[1] < 1) return fail(c, ICX_ERR_INVALID, "nelem must be positive");
  c->nx = nelem[0];
  c->ny = nelem[1];
  c->geo_order = geo_order;
  for (int d = 0; d < 2; ++d) { c->xmin[d] = xmin[d]; c->xmax[d] = xmax[d]; }
  for (int i = 0; i < 4; ++i) { c->bctype[i] = bctypes[i]; c->bcflag[i] = bcflags[i]; }
  int g = geo_order, nnx = c->nx * g + 1, nny = c->ny * g + 1;
  // node lattice, x fastest, equispaced over the full box (mesh.hpp:597-616)
  c->coord.assign((size_t)nnx * nny * 2, 0.0);
  for (int iy = 0; iy < nny; ++iy)
    for (int ix = 0; ix < nnx; ++ix) {
      size_t k = (size_t)ix + (size_t)nnx * iy;
      c->coord[2 * k] = xmin[0] + (xmax[0] - xmin[0]) * ix / (c->nx * g);
      c->coord[2 * k + 1] = xmin[1] + (xmax[1] - xmin[1]) * iy / (c->ny * g);
    }
  // element node lists, element (i, j) = i + nx j, local nodes dim 0 slowest (mesh.hpp:628-662)
  int ng = (g + 1) * (g + 1), E = c->nx * c->ny;
  c->el_nodes.assign((size_t)E * ng, 0);
  for (int e = 0; e < E; ++e) {
    int i = e % c->nx, j = e / c->nx;
    for (int k = 0; k < ng; ++k) {
      int k0 = k / (g + 1), k1 = k % (g + 1);
      c->el_nodes[(size_t)e * ng + k] = (i * g + k0) + nnx * (j * g + k1);
    }
  }
  // faces: interior per direction (left element index with i fastest), then
  // boundary (-, +) pairs per direction (mesh.hpp:674-892)
  c->faces.clear();
  auto vert = [&](int e, int fn, double s) {
    double xi[2];
    face_ref(fn, s, xi);
    int k0 = xi[0] < 0 ? 0 : g, k1 = xi[1] < 0 ? 0 : g;
    return c->el_nodes[(size_t)e * ng + k0 * (g + 1) + k1];
  };
  for (int idir = 0; idir < 2; ++idir) {
    if ((idir == 0 ? c->nx : c->ny) <= 1) continue;
    int ni = c->nx - (idir == 0), nj = c->ny - (idir == 1);
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        int L = i + c->nx * j, R = idir == 0 ? L + 1 : L + c->nx;
        int fnl = 2 + idir, fnr = idir;
        // orientation: 1 when the right face's first vertex is the left face's last
        int orient = (vert(R, fnr, -1.0) == vert(L, fnl, 1.0)) ? 1 : 0;
        int rec[7] = {L, R, fnl, fnr, orient, ICX_BC_INTERIOR, 0};
        c->faces.insert(c->faces.end(), rec, rec + 7);
      }
  }
  c->n_interior = (int)c->faces.size() / 7;
  for (int idim = 0; idim < 2; ++idim) {
    int nb = idim == 0 ? c->ny : c->nx;
    for (int t = 0; t < nb; ++t) {
      int LA = idim == 0 ? c->nx * t : t;
      int LB = idim == 0 ? c->nx * t + c->nx - 1 : t + c->nx * (c->ny - 1);
      int ra[7] = {LA, -1, idim, 0, 0, bctypes[idim], bcflags[idim]};
      int rb[7] = {LB, -1, idim + 2, 0, 0, bctypes[idim + 2], bcflags[idim + 2]};
      if (bctypes[idim] == ICX_BC_PERIODIC) {
        // a periodic pair's flags name each other's face index (mesh.hpp:857-866);
        // the faces stay boundary faces of their elements
        int fa = (int)c->faces.size() / 7;
        ra[6] = fa + 1;
        rb[6] = fa;
      }
      c->faces.insert(c->faces.end(), ra, ra + 7);
      c->faces.insert(c->faces.end(), rb, rb + 7);
    }
  }
  c->n_elem = c->nx * c->ny;
  c->el_level.resize(c->n_elem);
  c->el_i.resize(c->n_elem);
  c->el_j.resize(c->n_elem);
  c->el_grid.assign(c->n_elem, 0);
  for (int e = 0; e < c->n_elem; ++e) {
    c->el_i[e] = e % c->nx;
    c->el_j[e] = e / c->nx;
    c->el_level[e] = c->el_i[e] + c->el_j[e];
  }
  c->has_mesh = true;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_mesh_set_coords(icx_ctx* c, const double* xy) {
  if (!c || !xy || !c->has_mesh) return fail(c, ICX_ERR_INVALID, "mesh not created");
  std::memcpy(c->coord.data(), xy, sizeof(double) * c->coord.size());
  if (c->ready) {
    cudaSetDevice(c->device);
    return tabulate_and_geometry(c);
  }
  return ICX_OK;
}

icx_status icx_mesh_get_coords(const icx_ctx* c, double* xy) {
  if (!c || !xy || !c->has_mesh) return ICX_ERR_INVALID;
  std::memcpy(xy, c->coord.data(), sizeof(double) * c->coord.size());
  return ICX_OK;
}

icx_status icx_mesh_topology(const icx_ctx* c, int* conn, int* faces, int* n_interior) {
  if (!c || !c->has_mesh) return ICX_ERR_INVALID;
  if (conn) std::memcpy(conn, c->el_nodes.data(), sizeof(int) * c->el_nodes.size());
  if (faces) std::memcpy(faces, c->faces.data(), sizeof(int) * c->faces.size());
  if (n_interior) *n_interior = c->n_interior;
  return ICX_OK;
}

icx_status icx_fespace(icx_ctx* c, int basis_order) {
  if (!c || !c->has_mesh) return fail(c, ICX_ERR_INVALID, "mesh not created");
  if (basis_order < 1 || basis_order > icx::MAX_P)
    return fail(c, ICX_ERR_UNSUPPORTED, "basis order must be in 1..4");
  c->p = basis_order;
  c->basis = ICX_BASIS_LAGRANGE;
  c->has_space = true;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_fespace_basis(icx_ctx* c, int basis_order, int basis) {
  if (basis != ICX_BASIS_LAGRANGE && basis != ICX_BASIS_LEGENDRE) return fail(c, ICX_ERR_INVALID, "unknown basis");
  icx_status st = icx_fespace(c, basis_order);
  if (st == ICX_OK) c->basis = basis;
  return st;
}

icx_status icx_disc_burgers(icx_ctx* c, double mu, const double* a, const double* b) {
  if (!c || !a || !b) return fail(c, ICX_ERR_INVALID, "null argument");
  c->phys.pde = ICX_PDE_BURGERS;
  c->phys.mu = mu;
  c->phys.mu_t = mu;
  c->phys.spacetime = 0;
  for (int d = 0; d < 2; ++d) { c->phys.a[d] = a[d]; c->phys.b[d] = b[d]; }
  c->conv_flux = ICX_FLUX_UPWIND;
  c->has_disc = true;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_disc_spacetime_burgers(icx_ctx* c, double mu, double a, double b) {
  if (!c) return ICX_ERR_INVALID;
  c->phys.pde = ICX_PDE_BURGERS;
  c->phys.mu = mu;
  c->phys.mu_t = 0.0;
  c->phys.spacetime = 1;
  c->phys.a[0] = a;
  c->phys.b[0] = b;
  c->phys.a[1] = 1.0;  // time component of the flux: u
  c->phys.b[1] = 0.0;
  c->conv_flux = ICX_FLUX_UPWIND;
  c->has_disc = true;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_disc_navier_stokes(icx_ctx* c, double gamma, double Pr, double mu, int conv_flux) {
  if (!c) return ICX_ERR_INVALID;
  if (conv_flux != ICX_FLUX_VANLEER && conv_flux != ICX_FLUX_ROE)
    return fail(c, ICX_ERR_UNSUPPORTED, "Navier-Stokes convective flux: Van Leer or Roe");
  c->phys.ns_flux = conv_flux;
  c->phys.ns_viscous_wall = mu != 0.0;
  c->phys.ns_visc = 0;
  if (!(c->phys.Rgas > 0.0)) c->phys.Rgas = 287.052874;  // EoS::Rgas default (navier_stokes.hpp:338)
  c->phys.pde = ICX_PDE_NAVIER_STOKES;
  c->phys.gamma = gamma;
  c->phys.Pr = Pr;
  c->phys.ns_mu = mu;
  c->phys.inv_gamma = 1.0 / gamma;
  c->phys.inv_2gam2m1 = 1.0 / (2 * (gamma * gamma - 1));
  c->phys.mu_gamma_pr = mu * gamma / Pr;
  c->conv_flux = conv_flux;
  c->has_disc = true;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_disc_ns_boundary(icx_ctx* c, const double* wall_temperatures, int n_walls, double rho_inf,
                                double u_inf, const double u_direction[2], double T_inf, double Rgas) {
  if (!c) return ICX_ERR_INVALID;
  if (n_walls < 0 || n_walls > 8 || (n_walls > 0 && !wall_temperatures))
    return fail(c, ICX_ERR_INVALID, "wall temperatures: 0..8 values");
  if (!(Rgas > 0.0)) return fail(c, ICX_ERR_INVALID, "the gas constant must be positive");
  c->wall_T.assign(wall_temperatures, wall_temperatures + n_walls);
  c->phys.fs_rho = rho_inf;
  c->phys.fs_u[0] = u_direction ? u_direction[0] * u_inf : u_inf;
  c->phys.fs_u[1] = u_direction ? u_direction[1] * u_inf : 0.0;
  c->phys.fs_T = T_inf;
  c->phys.Rgas = Rgas;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_disc_ns_viscosity(icx_ctx* c, int kind, double mu_ratio, double T0_ratio, double Ts_ratio) {
  if (!c) return ICX_ERR_INVALID;
  if (!c->has_disc || c->phys.pde != ICX_PDE_NAVIER_STOKES)
    return fail(c, ICX_ERR_INVALID, "the viscosity law follows icx_disc_navier_stokes");
  if (kind == 0) {
    c->phys.ns_visc = 0;
    c->phys.ns_viscous_wall = c->phys.ns_mu != 0.0;
  } else if (kind == 1) {
    if (!(T0_ratio > 0.0) || !(Ts_ratio >= 0.0))
      return fail(c, ICX_ERR_INVALID, "Sutherland temperatures: T0_ratio > 0, Ts_ratio >= 0");
    c->phys.ns_visc = 1;
    c->phys.suth[0] = mu_ratio;
    c->phys.suth[1] = T0_ratio;
    c->phys.suth[2] = Ts_ratio;
    c->phys.ns_viscous_wall = 1;
  } else {
    return fail(c, ICX_ERR_INVALID, "viscosity law: 0 constant, 1 dimensionless Sutherland");
  }
  c->ready = false;
  return ICX_OK;
}

icx_status icx_disc_options(icx_ctx* c, int interior_penalty, double sigma_ic) {
  if (!c) return ICX_ERR_INVALID;
  c->phys.interior_penalty = interior_penalty;
  c->phys.sigma_ic = sigma_ic;
  c->ready = false;
  return ICX_OK;
}

static icx_status set_cb(icx_ctx* c, std::vector<icx_point_fn>& fns, std::vector<void*>& users, int flag,
                         icx_point_fn fn, void* user) {
  if (!c || flag < 0 || flag > 1024) return fail(c, ICX_ERR_INVALID, "bad boundary flag");
  if ((int)fns.size() <= flag) { fns.resize(flag + 1, nullptr); users.resize(flag + 1, nullptr); }
  fns[flag] = fn;
  users[flag] = user;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_disc_dirichlet(icx_ctx* c, int flag, icx_point_fn fn, void* user) {
  return set_cb(c, c->dirichlet_fn, c->dirichlet_user, flag, fn, user);
}
icx_status icx_disc_neumann(icx_ctx* c, int flag, icx_point_fn fn, void* user) {
  return set_cb(c, c->neumann_fn, c->neumann_user, flag, fn, user);
}
icx_status icx_disc_source(icx_ctx* c, icx_point_fn fn, void* user) {
  if (!c) return ICX_ERR_INVALID;
  c->source_fn = fn;
  c->source_user = user;
  c->ready = false;
  return ICX_OK;
}

icx_status icx_setup(icx_ctx* c) {
  if (!c || !c->has_mesh || !c->has_space || !c->has_disc)
    return fail(c, ICX_ERR_INVALID, "mesh, fespace and disc must be defined before setup");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
  // the solver buffers (element order, ILU pattern checks, CUDA graphs of the
  // GMRES steps) refer to the device tables rebuilt below
  icx::free_solver_work(c);
  free_dev(c->dm);
  DeviceMesh& dm = c->dm;
  int g = c->geo_order, P = c->p;
  dm.P = P;
  dm.G = g;
  dm.E = c->n_elem;
  dm.F = (int)c->faces.size() / 7;
  dm.Fi = c->n_interior;
  dm.Fb = dm.F - dm.Fi;
  dm.n_nodes = n_nodes(c);
  dm.nb = (P + 1) * (P + 1);
  dm.neq = c->phys.pde == ICX_PDE_BURGERS ? 1 : 4;
  dm.ng = (g + 1) * (g + 1);
  dm.nq1 = g + P;  // geometry order + basis order points per direction (reference_element.hpp:80, 240-245)
  dm.nqv = dm.nq1 * dm.nq1;
  dm.nqf = dm.nq1;
  // boundary kinds: PERIODIC, INLET and OUTLET have no implementation in
  // the reference's Navier-Stokes apply_bc (it logs "Unsupported BC" and
  // leaves the exterior state unset), so they are refused here
  if (c->phys.pde == ICX_PDE_NAVIER_STOKES)
    for (int i = 0; i < 4; ++i) {
      int b = c->bctype[i];
      if (b == ICX_BC_PERIODIC || b == 9 || b == 10 || b == ICX_BC_SPACETIME_PAST)
        return fail(c, ICX_ERR_UNSUPPORTED,
                    "Navier-Stokes periodic/inlet/outlet/spacetime boundaries are not implemented");
    }
  if (c->phys.pde == ICX_PDE_NAVIER_STOKES && c->phys.sigma_ic != 0.0) {
    // the Navier-Stokes diffusive flux defines no homogeneity tensor: the
    // reference skips the interface correction, so sigma_ic has no effect
  }
  // neither does the spacetime Burgers diffusion (burgers.hpp:414-474): the
  // kernels see sigma_ic = 0; SPACETIME_PAST faces without a connected past
  // slab contribute nothing, as in the reference without spacetime information
  if (c->phys.spacetime) c->phys.sigma_ic = 0.0;
  // DDG coefficients (conservation_law.hpp:511-538)
  c->phys.beta0 = std::pow(P + 1, 2);
  c->phys.beta1 = 1.0 / std::max((double)(2 * P * (P + 1)), 1.0);
  if (c->phys.interior_penalty) c->phys.beta1 = 0.0;

  Lagrange1D lb(P, c->basis), lg(g);
  double qx[16], qw[16];
  gauss_legendre(dm.nq1, qx, qw);
  // volume tabulation [nqv][nb][3] followed by the nqv weights
  std::vector<double> tvol((size_t)dm.nqv * dm.nb * 3 + dm.nqv);
  std::vector<double> tgvol((size_t)dm.nqv * dm.ng * 2);
  std::vector<double> tmp(std::max(dm.nb, dm.ng) * 6);
  for (int q0 = 0; q0 < dm.nq1; ++q0)
    for (int q1 = 0; q1 < dm.nq1; ++q1) {
      int q = q0 * dm.nq1 + q1;
      double xi[2] = {qx[q0], qx[q1]};
      tp_tab(lb, xi, tmp.data());
      for (int i = 0; i < dm.nb; ++i)
        for (int a = 0; a < 3; ++a) tvol[((size_t)q * dm.nb + i) * 3 + a] = tmp[i * 6 + a];
      tvol[(size_t)dm.nqv * dm.nb * 3 + q] = qw[q0] * qw[q1];
      tp_tab(lg, xi, tmp.data());
      for (int n = 0; n < dm.ng; ++n)
        for (int a = 0; a < 2; ++a) tgvol[((size_t)q * dm.ng + n) * 2 + a] = tmp[n * 6 + 1 + a];
    }
  // face tabulations for each local face and orientation
  std::vector<double> tface((size_t)8 * dm.nqf * dm.nb * 6), tgface((size_t)8 * dm.nqf * dm.ng * 6);
  for (int lf = 0; lf < 4; ++lf)
    for (int o = 0; o < 2; ++o)
      for (int q = 0; q < dm.nqf; ++q) {
        double xi[2];
        face_ref(lf, o ? -qx[q] : qx[q], xi);
        tp_tab(lb, xi, &tface[((size_t)(lf * 2 + o) * dm.nqf + q) * dm.nb * 6]);
        tp_tab(lg, xi, &tgface[((size_t)(lf * 2 + o) * dm.nqf + q) * dm.ng * 6]);
      }
  // 1D factors of the volume tabulation (sum factorisation): values, then
  // derivatives, of the p+1 Lagrange polynomials at the nq1 Gauss points
  std::vector<double> t1d((size_t)2 * dm.nq1 * (P + 1));
  for (int q = 0; q < dm.nq1; ++q) {
    double N[16], dN[16], d2N[16];
    lb.eval(qx[q], N, dN, d2N);
    for (int i = 0; i <= P; ++i) {
      t1d[(size_t)q * (P + 1) + i] = N[i];
      t1d[(size_t)(dm.nq1 + q) * (P + 1) + i] = dN[i];
    }
  }
  std::vector<double> tfphi((size_t)8 * dm.nqf * dm.nb);
  for (size_t k = 0; k < tfphi.size(); ++k) tfphi[k] = tface[k * 6];
  // face tabulation as 1D factors: the fixed coordinate of local face lf is
  // xi_(lf & 1) = -1 (lf < 2) or +1, the other follows the face point
  std::vector<double> tf1d((size_t)4 * (P + 1) * 3 + (size_t)8 * dm.nqf * (P + 1) * 3);
  for (int lf = 0; lf < 4; ++lf) {
    double N[16], dN[16], d2N[16];
    lb.eval(lf < 2 ? -1.0 : 1.0, N, dN, d2N);
    for (int k = 0; k <= P; ++k) {
      double* o = &tf1d[((size_t)lf * (P + 1) + k) * 3];
      o[0] = N[k]; o[1] = dN[k]; o[2] = d2N[k];
    }
    for (int o = 0; o < 2; ++o)
      for (int q = 0; q < dm.nqf; ++q) {
        double xi[2];
        face_ref(lf, o ? -qx[q] : qx[q], xi);
        lb.eval(xi[1 - (lf & 1)], N, dN, d2N);
        for (int j = 0; j <= P; ++j) {
          double* t = &tf1d[(size_t)4 * (P + 1) * 3 + ((((size_t)lf * 2 + o) * dm.nqf + q) * (P + 1) + j) * 3];
          t[0] = N[j]; t[1] = dN[j]; t[2] = d2N[j];
        }
      }
  }
  std::vector<double> tgcen(dm.ng);
  {
    double xi0[2] = {0.0, 0.0};
    tp_tab(lg, xi0, tmp.data());
    for (int n = 0; n < dm.ng; ++n) tgcen[n] = tmp[n * 6];
  }
  std::vector<double> qwf(qw, qw + dm.nqf);
  // face records with boundary index; element-to-face adjacency
  std::vector<int> finfo((size_t)dm.F * 8);
  std::vector<int> elf((size_t)dm.E * 4, -1), els((size_t)dm.E * 4, 0);
  for (int f = 0; f < dm.F; ++f) {
    const int* F = &c->faces[7 * f];
    for (int a = 0; a < 7; ++a) finfo[8 * f + a] = F[a];
    finfo[8 * f + 7] = f >= dm.Fi ? f - dm.Fi : -1;
    elf[F[0] * 4 + F[2]] = f;
    els[F[0] * 4 + F[2]] = 0;
    if (F[1] >= 0) { elf[F[1] * 4 + F[3]] = f; els[F[1] * 4 + F[3]] = 1; }
  }
  // block pattern and face block positions (reference sparsity: element
  // blocks couple to themselves and face neighbours)
  std::vector<int> rowptr(dm.E + 1, 0), colidx, diag(dm.E), fblk((size_t)dm.F * 4, -1);
  for (int e = 0; e < dm.E; ++e) {
    // the element and its face neighbours, ascending
    int cols[5], nc = 0;
    cols[nc++] = e;
    for (int lf = 0; lf < 4; ++lf) {
      int f = elf[(size_t)e * 4 + lf];
      if (f < 0) continue;
      int L = c->faces[7 * f], R = c->faces[7 * f + 1];
      if (R >= 0) cols[nc++] = (L == e) ? R : L;
    }
    std::sort(cols, cols + nc);
    for (int k = 0; k < nc; ++k) {
      if (cols[k] == e) diag[e] = (int)colidx.size();
      colidx.push_back(cols[k]);
    }
    rowptr[e + 1] = (int)colidx.size();
  }
  auto find_blk = [&](int r, int col) {
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k)
      if (colidx[k] == col) return k;
    return -1;
  };
  for (int f = 0; f < dm.F; ++f) {
    int L = c->faces[7 * f], R = c->faces[7 * f + 1];
    fblk[4 * f + 0] = diag[L];
    if (R >= 0) {
      fblk[4 * f + 1] = find_blk(L, R);
      fblk[4 * f + 2] = find_blk(R, L);
      fblk[4 * f + 3] = diag[R];
    }
  }
  dm.nnzb = (int)colidx.size();

  std::vector<cudaError_t> errs;
  errs.push_back(upload(&dm.el_nodes, c->el_nodes));
  errs.push_back(upload(&dm.face_info, finfo));
  errs.push_back(upload(&dm.el_face, elf));
  errs.push_back(upload(&dm.el_side, els));
  {
    std::vector<int> fso((size_t)dm.E * 4, 0);
    for (size_t k = 0; k < fso.size(); ++k) {
      int f = elf[k], side = els[k];
      int o = side ? c->faces[7 * f + 4] : 0;
      fso[k] = f * 4 + side + 2 * o;
    }
    errs.push_back(upload(&dm.el_fso, fso));
  }
  errs.push_back(upload(&dm.tab_vol, tvol));
  errs.push_back(upload(&dm.tab_face, tface));
  errs.push_back(upload(&dm.tab_1d, t1d));
  errs.push_back(upload(&dm.tab_fphi, tfphi));
  errs.push_back(upload(&dm.tab_f1d, tf1d));
  errs.push_back(upload(&dm.tab_gvol, tgvol));
  errs.push_back(upload(&dm.tab_gface, tgface));
  errs.push_back(upload(&dm.tab_gcen, tgcen));
  errs.push_back(upload(&dm.qw_face, qwf));
  errs.push_back(upload(&dm.bsr_rowptr, rowptr));
  errs.push_back(upload(&dm.bsr_colidx, colidx));
  errs.push_back(upload(&dm.bsr_diag, diag));
  errs.push_back(upload(&dm.face_blk, fblk));
  errs.push_back(cudaMalloc((void**)&dm.vgeo, sizeof(double) * 5 * dm.E * dm.nqv));
  errs.push_back(cudaMalloc((void**)&dm.fgeo, sizeof(double) * icx::NFACE_GEO * dm.F * dm.nqf));
  errs.push_back(cudaMalloc((void**)&dm.face_flux, sizeof(double) * (size_t)dm.F * dm.nqf * dm.neq));
  errs.push_back(cudaMalloc((void**)&dm.face_grad, sizeof(double) * (size_t)dm.F * 2 * dm.nqf * dm.neq * 2));
  for (cudaError_t e2 : errs)
    if (e2 != cudaSuccess) return cuda_fail(c, e2, "device table allocation");
  icx_status st = tabulate_and_geometry(c);
  if (st != ICX_OK) return st;
  c->ready = true;
  return ICX_OK;
}

icx_status icx_get_layout(const icx_ctx* c, icx_layout_info* info) {
  if (!c || !info || !c->ready) return ICX_ERR_INVALID;
  const DeviceMesh& dm = c->dm;
  info->n_elem = dm.E;
  info->nbasis = dm.nb;
  info->neq = dm.neq;
  info->block_size = dm.nb * dm.neq;
  info->n_dof = (long long)dm.E * dm.nb * dm.neq;
  info->n_faces = dm.F;
  info->n_interior_faces = dm.Fi;
  info->n_nodes = dm.n_nodes;
  info->nnz_blocks = dm.nnzb;
  info->nq_vol = dm.nqv;
  info->nq_face = dm.nqf;
  return ICX_OK;
}

icx_status icx_form_residual(icx_ctx* c, const double* d_u, double* d_res, void* stream) {
  if (!c || !c->ready) return fail(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !d_res) return fail(c, ICX_ERR_INVALID, "null device pointer");
  cudaError_t e = icx::launch_residual(c->dm, c->phys, d_u, d_res, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "residual kernels");
  return ICX_OK;
}

icx_status icx_form_residual_timed(icx_ctx* c, const double* d_u, double* d_res, void* stream, double* ms_face,
                                   double* ms_volume) {
  if (!c || !c->ready) return fail(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !d_res) return fail(c, ICX_ERR_INVALID, "null device pointer");
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t ev[3];
  for (auto& e : ev) cudaEventCreate(&e);
  cudaEventRecord(ev[0], s);
  cudaError_t e = icx::launch_residual(c->dm, c->phys, d_u, d_res, s, ev[1]);
  cudaEventRecord(ev[2], s);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev[2]);
  float a = 0.f, b = 0.f;
  cudaEventElapsedTime(&a, ev[0], ev[1]);
  cudaEventElapsedTime(&b, ev[1], ev[2]);
  for (auto& x : ev) cudaEventDestroy(x);
  if (e != cudaSuccess) return cuda_fail(c, e, "residual kernels");
  if (ms_face) *ms_face = a;
  if (ms_volume) *ms_volume = b;
  return ICX_OK;
}

icx_status icx_basis_node_coords(const icx_ctx* c, double* xy) {
  if (!c || !xy || !c->has_mesh || !c->has_space) return ICX_ERR_INVALID;
  if (c->basis != ICX_BASIS_LAGRANGE) return ICX_ERR_UNSUPPORTED;  // a modal basis has no nodes
  Lagrange1D lb(c->p), lg(c->geo_order);
  int n = c->p + 1, E = c->n_elem;
  for (int e = 0; e < E; ++e)
    for (int i0 = 0; i0 < n; ++i0)
      for (int i1 = 0; i1 < n; ++i1) {
        double xi[2] = {lb.xi[i0], lb.xi[i1]};
        el_point(c, lg, e, xi, xy + ((size_t)(e * n * n + i0 * n + i1)) * 2);
      }
  return ICX_OK;
}

icx_status icx_jacobian_pattern(const icx_ctx* c, int* rowptr, int* colidx) {
  if (!c || !c->ready || !rowptr || !colidx) return ICX_ERR_INVALID;
  cudaError_t e = cudaMemcpy(rowptr, c->dm.bsr_rowptr, sizeof(int) * (c->dm.E + 1), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(colidx, c->dm.bsr_colidx, sizeof(int) * c->dm.nnzb, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? ICX_OK : ICX_ERR_CUDA;
}

}  // extern "C"
