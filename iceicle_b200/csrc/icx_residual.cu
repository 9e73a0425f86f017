// DG residual on the GPU: geometry factors, face numerical fluxes and the
// element volume integral with the face lifting, for 2D quadrilaterals of
// geometry order G and Lagrange order P.
//
// Structure (form_residual, src/solvers/include/iceicle/form_residual.hpp:56-268):
//   geometry kernels  - once per mesh / node update: per volume point
//                       J^-1 and w*max(det J, 0); per face point the unit
//                       normal, w*sqrt(g), the DDG distance and both sides'
//                       J^-1 and transformation Hessians.
//   face_flux_kernel  - one thread per face quadrature point evaluates the
//                       convective + DDG viscous numerical flux
//                       (trace_integral / boundaryIntegral, conservation_law.hpp:434-1176)
//                       and stores (f_visc - f_adv) * w * sqrt(g).
//   vol_lift_kernel   - one CTA per group of elements: volume integral
//                       (domain_integral, conservation_law.hpp:244-314), then
//                       lifts the stored face fluxes of its four faces onto
//                       its test functions. Every residual entry is written
//                       exactly once: no atomics and no zero fill.
#include <cfloat>
#include <cstdio>

#include "icx_internal.h"
#include "icx_dg.cuh"

namespace icx {


__constant__ double c_dxi_ds[4][2] = {{0.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}};

// ---------------------------------------------------------------- geometry
template <int P, int G>
__global__ void geo_vol_kernel(DeviceMesh dm) {
  constexpr int NQ1 = G + P, NQV = NQ1 * NQ1, NG = (G + 1) * (G + 1);
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= dm.E * NQV) return;
  int e = k / NQV, q = k - e * NQV;
  double J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int n = 0; n < NG; ++n) {
    int gn = dm.el_nodes[e * NG + n];
    double x0 = dm.coord[2 * gn], x1 = dm.coord[2 * gn + 1];
    double d0 = dm.tab_gvol[(q * NG + n) * 2], d1 = dm.tab_gvol[(q * NG + n) * 2 + 1];
    J[0][0] += d0 * x0; J[0][1] += d1 * x0;
    J[1][0] += d0 * x1; J[1][1] += d1 * x1;
  }
  double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  double ds = (det == 0.0) ? 1.0 : det;
  int nq = dm.E * NQV;
  dm.vgeo[0 * nq + k] = J[1][1] / ds;
  dm.vgeo[1 * nq + k] = -J[0][1] / ds;
  dm.vgeo[2 * nq + k] = -J[1][0] / ds;
  dm.vgeo[3 * nq + k] = J[0][0] / ds;
  // quadrature weight is folded into the volume tabulation's 4th component
  double w = dm.tab_vol[(size_t)dm.nqv * dm.nb * 3 + q];
  dm.vgeo[4 * nq + k] = fmax(0.0, det) * w;
}

// x, J and the transformation Hessian of element e at tabulated face point t
template <int NG>
__device__ inline void face_side_geo(const DeviceMesh& dm, int e, const double* tab, double x[2], double J[2][2],
                                     double H[2][3]) {
  x[0] = x[1] = 0.0;
  J[0][0] = J[0][1] = J[1][0] = J[1][1] = 0.0;
  H[0][0] = H[0][1] = H[0][2] = H[1][0] = H[1][1] = H[1][2] = 0.0;
#pragma unroll
  for (int n = 0; n < NG; ++n) {
    int gn = dm.el_nodes[e * NG + n];
    double xn[2] = {dm.coord[2 * gn], dm.coord[2 * gn + 1]};
    const double* t = tab + n * 6;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      x[i] += t[0] * xn[i];
      J[i][0] += t[1] * xn[i];
      J[i][1] += t[2] * xn[i];
      H[i][0] += t[3] * xn[i];
      H[i][1] += t[4] * xn[i];
      H[i][2] += t[5] * xn[i];
    }
  }
}

template <int NG>
__device__ inline void centroid(const DeviceMesh& dm, int e, double c[2]) {
  c[0] = c[1] = 0.0;
#pragma unroll
  for (int n = 0; n < NG; ++n) {
    int gn = dm.el_nodes[e * NG + n];
    c[0] += dm.tab_gcen[n] * dm.coord[2 * gn];
    c[1] += dm.tab_gcen[n] * dm.coord[2 * gn + 1];
  }
}

__device__ inline void store_jinv(double* fgeo, int nfq, int k, int off, const double J[2][2]) {
  double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  double ds = (det == 0.0) ? 1.0 : det;
  fgeo[(off + 0) * nfq + k] = J[1][1] / ds;
  fgeo[(off + 1) * nfq + k] = -J[0][1] / ds;
  fgeo[(off + 2) * nfq + k] = -J[1][0] / ds;
  fgeo[(off + 3) * nfq + k] = J[0][0] / ds;
}

template <int P, int G>
__global__ void geo_face_kernel(DeviceMesh dm) {
  constexpr int NQF = G + P, NG = (G + 1) * (G + 1);
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= dm.F * NQF) return;
  int f = k / NQF, q = k - f * NQF;
  const int* fi = dm.face_info + 8 * f;
  int L = fi[0], R = fi[1], fnl = fi[2], fnr = fi[3], orient = fi[4];
  double x[2], J[2][2], H[2][3];
  face_side_geo<NG>(dm, L, dm.tab_gface + ((size_t)((fnl * 2 + 0) * NQF + q) * NG) * 6, x, J, H);
  double t0 = J[0][0] * c_dxi_ds[fnl][0] + J[0][1] * c_dxi_ds[fnl][1];
  double t1 = J[1][0] * c_dxi_ds[fnl][0] + J[1][1] * c_dxi_ds[fnl][1];
  double sqrtg = sqrt(t0 * t0 + t1 * t1);
  double nn = sqrt(t1 * t1 + t0 * t0);
  double n0 = t1 / nn, n1 = -t0 / nn;
  int nfq = dm.F * NQF;
  double* g = dm.fgeo;
  g[FG_N0 * nfq + k] = n0;
  g[FG_N1 * nfq + k] = n1;
  g[FG_WSQ * nfq + k] = dm.qw_face[q] * sqrtg;
  store_jinv(g, nfq, k, FG_JIL, J);
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int a = 0; a < 3; ++a) g[(FG_HL + 3 * m + a) * nfq + k] = H[m][a];
  double cL[2];
  centroid<NG>(dm, L, cL);
  double h = 0.0;
  if (R >= 0) {
    double xr[2], JR[2][2], HR[2][3], cR[2];
    face_side_geo<NG>(dm, R, dm.tab_gface + ((size_t)((fnr * 2 + orient) * NQF + q) * NG) * 6, xr, JR, HR);
    centroid<NG>(dm, R, cR);
    h = n0 * ((x[0] - cL[0]) + (cR[0] - x[0])) + n1 * ((x[1] - cL[1]) + (cR[1] - x[1]));
    store_jinv(g, nfq, k, FG_JIR, JR);
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int a = 0; a < 3; ++a) g[(FG_HR + 3 * m + a) * nfq + k] = HR[m][a];
  } else {
    h = fabs(n0 * (x[0] - cL[0])) + fabs(n1 * (x[1] - cL[1]));
#pragma unroll
    for (int a = 0; a < 10; ++a) g[(FG_JIR + a) * nfq + k] = 0.0;
  }
  g[FG_H * nfq + k] = copysign(fmax(fabs(h), DBL_EPSILON), h);
}

// ------------------------------------------------------------- face fluxes
template <int PDE, int P, int G, bool DDG>
__global__ void face_flux_kernel(DeviceMesh dm, PhysParams pp, const double* __restrict__ u) {
  using C = Cfg<PDE, P, G>;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= dm.F * C::NQF) return;
  int f = k / C::NQF, q = k - f * C::NQF;
  const int* fi = dm.face_info + 8 * f;
  int L = fi[0], R = fi[1];
  double out[C::NEQ], gq[4];
  face_point_flux<PDE, P, G, DDG>(dm, pp, f, q, u + (size_t)L * C::BS, u + (size_t)(R >= 0 ? R : L) * C::BS, out,
                                  gq);
#pragma unroll
  for (int eq = 0; eq < C::NEQ; ++eq) dm.face_flux[(size_t)k * C::NEQ + eq] = out[eq];
  if (Phys<PDE>::has_ic && pp.sigma_ic != 0.0) {
    // layout [F][side][NQF][NEQ=1][2]
    double* fg = dm.face_grad + (size_t)f * 2 * C::NQF * 2;
    fg[(0 * C::NQF + q) * 2 + 0] = gq[0];
    fg[(0 * C::NQF + q) * 2 + 1] = gq[1];
    fg[(1 * C::NQF + q) * 2 + 0] = gq[2];
    fg[(1 * C::NQF + q) * 2 + 1] = gq[3];
  }
}

// ----------------------------------------------------- volume + face lifting
template <int PDE, int P, int G>
struct VolCfg {
  using C = Cfg<PDE, P, G>;
  static constexpr int THREADS = 256;
  static constexpr int EPB_RAW = THREADS / C::NQV;
  static constexpr int EPB = EPB_RAW < 1 ? 1 : EPB_RAW;
  static constexpr int TAB = C::NQV * C::NB * 3;                     // doubles
  static constexpr int PER_EL = C::BS + C::NQV * C::NEQ * 3;          // coef + G + S
  static constexpr size_t SMEM = sizeof(double) * (TAB + EPB * PER_EL);
};

template <int PDE, int P, int G>
__global__ void __launch_bounds__(256) vol_lift_kernel(DeviceMesh dm, PhysParams pp, const double* __restrict__ u,
                                                       double* __restrict__ res) {
  using C = Cfg<PDE, P, G>;
  using V = VolCfg<PDE, P, G>;
  constexpr int NEQ = C::NEQ, NB = C::NB, BS = C::BS, NQV = C::NQV, NQF = C::NQF, EPB = V::EPB;
  extern __shared__ double smem[];
  double* s_tab = smem;                          // [NQV][NB][3]
  double* s_coef = s_tab + V::TAB;               // [EPB][BS]
  double* s_G = s_coef + EPB * BS;               // [EPB][NQV][NEQ][2]
  double* s_S = s_G + EPB * NQV * NEQ * 2;       // [EPB][NQV][NEQ]
  const int e0 = blockIdx.x * EPB;
  const int ne = min(EPB, dm.E - e0);
  const int tid = threadIdx.x;
  for (int t = tid; t < V::TAB; t += blockDim.x) s_tab[t] = dm.tab_vol[t];
  // element coefficient tiles are contiguous in the reference layout
  const double* ublk = u + (size_t)e0 * BS;
  for (int t = tid; t < ne * BS; t += blockDim.x) s_coef[t] = ublk[t];
  __syncthreads();

  const int nq = dm.E * NQV;
  const bool has_src = dm.src != nullptr;
  for (int t = tid; t < ne * NQV; t += blockDim.x) {
    int el = t / NQV, q = t - el * NQV;
    int e = e0 + el;
    const double* cf = s_coef + el * BS;
    const double* tb = s_tab + q * NB * 3;
    double uq[NEQ], gxi[NEQ][2];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) { uq[eq] = 0.0; gxi[eq][0] = gxi[eq][1] = 0.0; }
#pragma unroll 4
    for (int i = 0; i < NB; ++i) {
      double phi = tb[i * 3], d0 = tb[i * 3 + 1], d1 = tb[i * 3 + 2];
#pragma unroll
      for (int eq = 0; eq < NEQ; ++eq) {
        double c = cf[i * NEQ + eq];
        uq[eq] += c * phi;
        gxi[eq][0] += c * d0;
        gxi[eq][1] += c * d1;
      }
    }
    size_t kq = (size_t)e * NQV + q;
    double Ji[4] = {dm.vgeo[0 * nq + kq], dm.vgeo[1 * nq + kq], dm.vgeo[2 * nq + kq], dm.vgeo[3 * nq + kq]};
    double wd = dm.vgeo[4 * nq + kq];
    double gx[2 * NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq)
#pragma unroll
      for (int d = 0; d < 2; ++d) gx[eq * 2 + d] = gxi[eq][0] * Ji[0 * 2 + d] + gxi[eq][1] * Ji[1 * 2 + d];
    double F[2 * NEQ];
    Phys<PDE>::flux(pp, uq, gx, F);
    double* Gq = s_G + (el * NQV + q) * NEQ * 2;
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq)
#pragma unroll
      for (int kk = 0; kk < 2; ++kk)
        Gq[eq * 2 + kk] = (F[eq * 2 + 0] * Ji[kk * 2 + 0] + F[eq * 2 + 1] * Ji[kk * 2 + 1]) * wd;
    double* Sq = s_S + (el * NQV + q) * NEQ;
    if (has_src) {
#pragma unroll
      for (int eq = 0; eq < NEQ; ++eq) Sq[eq] = -dm.src[kq * NEQ + eq] * wd;
    }
  }
  __syncthreads();

  const bool ic = Phys<PDE>::has_ic && pp.sigma_ic != 0.0;
  for (int t = tid; t < ne * BS; t += blockDim.x) {
    int el = t / BS, r = t - el * BS;
    int i = r / NEQ, eq = r - i * NEQ;
    int e = e0 + el;
    const double* Gq = s_G + el * NQV * NEQ * 2;
    double acc = 0.0;
#pragma unroll 5
    for (int q = 0; q < NQV; ++q) {
      const double* tb = s_tab + (q * NB + i) * 3;
      acc += tb[1] * Gq[(q * NEQ + eq) * 2 + 0] + tb[2] * Gq[(q * NEQ + eq) * 2 + 1];
    }
    if (has_src) {
      const double* Sq = s_S + el * NQV * NEQ;
#pragma unroll 5
      for (int q = 0; q < NQV; ++q) acc += s_tab[(q * NB + i) * 3] * Sq[q * NEQ + eq];
    }
#pragma unroll
    for (int lf = 0; lf < 4; ++lf) {
      int fidx = dm.el_face[e * 4 + lf];
      int side = dm.el_side[e * 4 + lf];
      int o = side ? dm.face_info[8 * fidx + 4] : 0;
      const double* tf = dm.tab_face + ((size_t)(lf * 2 + o) * NQF * NB + i) * 6;
      const double* ff = dm.face_flux + (size_t)fidx * NQF * NEQ + eq;
      double s = 0.0;
#pragma unroll
      for (int qf = 0; qf < NQF; ++qf) s += tf[(size_t)qf * NB * 6] * ff[qf * NEQ];
      acc += side ? -s : s;
      if (ic) {
        const double* fg = dm.face_grad + ((size_t)(fidx * 2 + side) * NQF) * 2;
        double sg = 0.0;
#pragma unroll
        for (int qf = 0; qf < NQF; ++qf)
          sg += tf[(size_t)qf * NB * 6 + 1] * fg[qf * 2 + 0] + tf[(size_t)qf * NB * 6 + 2] * fg[qf * 2 + 1];
        acc -= sg;
      }
    }
    res[(size_t)e * BS + r] = acc;
  }
}

// --------------------------------------------------------------- launchers
template <int P, int G>
static cudaError_t geometry_pg(const DeviceMesh& dm, cudaStream_t s) {
  constexpr int NQ1 = G + P;
  int nv = dm.E * NQ1 * NQ1, nf = dm.F * NQ1;
  geo_vol_kernel<P, G><<<(nv + 255) / 256, 256, 0, s>>>(dm);
  geo_face_kernel<P, G><<<(nf + 255) / 256, 256, 0, s>>>(dm);
  return cudaGetLastError();
}

cudaError_t launch_geometry(const DeviceMesh& dm, cudaStream_t s) {
#define ICX_GEO_CASE(PP, GG) \
  if (dm.P == PP && dm.G == GG) return geometry_pg<PP, GG>(dm, s);
  ICX_GEO_CASE(1, 1) ICX_GEO_CASE(2, 1) ICX_GEO_CASE(3, 1) ICX_GEO_CASE(4, 1)
  ICX_GEO_CASE(1, 2) ICX_GEO_CASE(2, 2) ICX_GEO_CASE(3, 2) ICX_GEO_CASE(4, 2)
#undef ICX_GEO_CASE
  return cudaErrorInvalidValue;
}

template <int PDE, int P, int G>
static cudaError_t residual_pg(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                               cudaStream_t s, cudaEvent_t mid) {
  using C = Cfg<PDE, P, G>;
  using V = VolCfg<PDE, P, G>;
  int nf = dm.F * C::NQF;
  if (pp.beta1 != 0.0)
    face_flux_kernel<PDE, P, G, true><<<(nf + 127) / 128, 128, 0, s>>>(dm, pp, u);
  else
    face_flux_kernel<PDE, P, G, false><<<(nf + 127) / 128, 128, 0, s>>>(dm, pp, u);
  if (mid) cudaEventRecord(mid, s);
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(vol_lift_kernel<PDE, P, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)V::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  int nblk = (dm.E + V::EPB - 1) / V::EPB;
  vol_lift_kernel<PDE, P, G><<<nblk, V::THREADS, V::SMEM, s>>>(dm, pp, u, res);
  return cudaGetLastError();
}

cudaError_t launch_residual(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                            cudaStream_t s, cudaEvent_t mid) {
#define ICX_RES_CASE(PDE, PP, GG) \
  if (pp.pde == PDE && dm.P == PP && dm.G == GG) return residual_pg<PDE, PP, GG>(dm, pp, u, res, s, mid);
  ICX_RES_CASE(0, 1, 1) ICX_RES_CASE(0, 2, 1) ICX_RES_CASE(0, 3, 1) ICX_RES_CASE(0, 4, 1)
  ICX_RES_CASE(0, 1, 2) ICX_RES_CASE(0, 2, 2) ICX_RES_CASE(0, 3, 2) ICX_RES_CASE(0, 4, 2)
  ICX_RES_CASE(1, 1, 1) ICX_RES_CASE(1, 2, 1) ICX_RES_CASE(1, 3, 1) ICX_RES_CASE(1, 4, 1)
  ICX_RES_CASE(1, 1, 2) ICX_RES_CASE(1, 2, 2) ICX_RES_CASE(1, 3, 2) ICX_RES_CASE(1, 4, 2)
#undef ICX_RES_CASE
  return cudaErrorInvalidValue;
}

}  // namespace icx
