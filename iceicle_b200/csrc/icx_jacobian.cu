// Finite-difference Jacobian straight into BSR (form_petsc_jacobian_fd,
// src/solvers/include/iceicle/form_petsc_jacobian.hpp:55-317), with the
// reference's perturbation scheme:
//   * faces: every DOF of a side is perturbed by eps_f = max(eps, eps *
//     max(|R_L^f|_2, |R_R^f|_2)) where R^f are that face's own contributions to
//     the two elements' residuals (boundary faces: |R_L^f|_2), and the face's
//     flux is re-evaluated: J(:, c) += (R^f(u + eps_f e_c) - R^f(u)) / eps_f
//     (FJ:97-285, fd_utils.hpp:11-14);
//   * volume: flux-level FD at each quadrature point with
//     eps_q = max(sqrt(eps), sqrt(eps) |F|_F) over u and grad u, contracted
//     analytically with the basis (domain_integral_jacobian,
//     conservation_law.hpp:316-432).
//
// FP32 form (T = float): coefficient tiles, metrics, tabulations and fluxes
// rounded to FP32 and every product, sum and difference taken in FP32, with
// eps = sqrt(FLT_EPSILON) in place of sqrt(DBL_EPSILON) in both schemes; the
// blocks are written as FP32. The FP64 form is this kernel with T = double.
//
// Element-centric: one CTA per element e perturbs e's own DOFs only. It owns
// the diagonal block (volume + the four faces' e-e couplings) and, for each
// face with a neighbour n, the block (n, e) — the neighbour's residual with
// respect to e's DOFs. Every block of the pattern therefore has exactly one
// writer: no atomics, no zero fill.
#include <cfloat>

#include "icx_dg.cuh"
#include "icx_blockrow.cuh"

namespace icx {

template <int PDE, int P, int G, class T = double>
struct JacCfg {
  using C = Cfg<PDE, P, G>;
  static constexpr int THREADS = 256;
  static constexpr int NEQ = C::NEQ, NB = C::NB, BS = C::BS, NQF = C::NQF, NQV = C::NQV;
  static constexpr int NST = NEQ * 7;           // side state: u, grad, Hessian
  static constexpr int NFP = 24;                // FacePt scalars
  static constexpr int IC = Phys<PDE>::has_ic ? 1 : 0;
  // shared memory layout, in scalars of type T
  static constexpr int O_COEF = 0;                                   // [5][BS]
  static constexpr int O_FP = O_COEF + 5 * BS;                       // [4][NQF] FacePt
  static constexpr int O_FST = O_FP + 4 * NQF * NFP;                 // [4][NQF][2][NST]
  static constexpr int O_FQB = O_FST + 4 * NQF * 2 * NST;            // [4][NQF][NEQ]
  static constexpr int O_GQB = O_FQB + 4 * NQF * NEQ;                // [4][NQF][4]
  static constexpr int O_DFQ = O_GQB + IC * 4 * NQF * 4;             // [BS][4][NQF][NEQ]
  static constexpr int O_DGQ = O_DFQ + BS * 4 * NQF * NEQ;           // [BS][4][NQF][4]
  static constexpr int O_UQ = O_DGQ + IC * BS * 4 * NQF * 4;         // [NQV][NEQ]
  static constexpr int O_GQ = O_UQ + NQV * NEQ;                      // [NQV][NEQ][2]
  static constexpr int O_FB = O_GQ + NQV * NEQ * 2;                  // [NQV][NEQ][2]
  static constexpr int O_EPSQ = O_FB + NQV * NEQ * 2;                // [NQV]
  static constexpr int O_DFDU = O_EPSQ + NQV;                        // [NQV][NEQ][2][NEQ]
  static constexpr int O_DFDG = O_DFDU + NQV * NEQ * 2 * NEQ;        // [NQV][NEQ][2][NEQ][2]
  static constexpr int O_GPHI = O_DFDG + NQV * NEQ * 2 * NEQ * 2;    // [NQV][NB][2]
  static constexpr int O_WD = O_GPHI + NQV * NB * 2;                 // [NQV]
  static constexpr int O_EPSF = O_WD + NQV;                          // [4]
  static constexpr int TOTAL = O_EPSF + 4;
  static constexpr size_t SMEM = sizeof(T) * TOTAL;
  static_assert(SMEM <= 227 * 1024, "Jacobian tile exceeds the shared memory of one CTA");
};

template <class T>
__device__ inline void fp_store(T* s, const FacePtT<T>& p) {
  s[0] = p.n[0]; s[1] = p.n[1]; s[2] = p.wsq; s[3] = p.h;
#pragma unroll
  for (int a = 0; a < 4; ++a) { s[4 + a] = p.JiL[a]; s[14 + a] = p.JiR[a]; }
#pragma unroll
  for (int a = 0; a < 6; ++a) { s[8 + a] = p.HL[a]; s[18 + a] = p.HR[a]; }
}
template <class T>
__device__ inline void fp_load(const T* s, FacePtT<T>& p) {
  p.n[0] = s[0]; p.n[1] = s[1]; p.wsq = s[2]; p.h = s[3];
#pragma unroll
  for (int a = 0; a < 4; ++a) { p.JiL[a] = s[4 + a]; p.JiR[a] = s[14 + a]; }
#pragma unroll
  for (int a = 0; a < 6; ++a) { p.HL[a] = s[8 + a]; p.HR[a] = s[18 + a]; }
}

template <int PDE, int P, int G, bool DDG, class T>
__global__ void __launch_bounds__(256) jac_elem_kernel(DeviceMesh dm, PhysParams pp_in, const double* __restrict__ u,
                                                        T* __restrict__ vals, double eps_in) {
  // every face of the element joins it to the same problem: one parameter set
  const PhysParams pp = elem_params<PDE>(dm, pp_in, blockIdx.x);
  using J = JacCfg<PDE, P, G, T>;
  constexpr int NEQ = J::NEQ, NB = J::NB, BS = J::BS, NQF = J::NQF, NQV = J::NQV, NST = J::NST;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* sm = reinterpret_cast<T*>(sm_raw);
  const int e = blockIdx.x;
  const int tid = threadIdx.x;
  const bool ic = Phys<PDE>::has_ic && pp.sigma_ic != 0.0;
  const T sqeps = sizeof(T) == sizeof(double) ? T(sqrt(DBL_EPSILON)) : T(sqrtf(FLT_EPSILON));
  const T eps = T(eps_in);

  // per local face: face index, e's side, neighbour, tabulation slots
  int f_[4], side_[4], nbr_[4], oe_[4], lfn_[4], on_[4], bct_[4], bidx_[4];
#pragma unroll
  for (int lf = 0; lf < 4; ++lf) {
    int f = dm.el_face[e * 4 + lf];
    const int* fi = dm.face_info + 8 * f;
    int s = dm.el_side[e * 4 + lf];
    f_[lf] = f;
    side_[lf] = s;
    nbr_[lf] = fi[1] < 0 ? -1 : (s == 0 ? fi[1] : fi[0]);
    oe_[lf] = s ? fi[4] : 0;                  // orientation of e's tabulation
    lfn_[lf] = s ? fi[2] : fi[3];             // neighbour's local face number
    on_[lf] = s ? 0 : fi[4];                  // orientation of the neighbour's tabulation
    bct_[lf] = fi[5];
    bidx_[lf] = fi[7];
  }

  // ---- load coefficient tiles: [0] = e, [1 + lf] = neighbour across lf
  for (int t = tid; t < 5 * BS; t += blockDim.x) {
    int slot = t / BS, r = t - slot * BS;
    int el = slot == 0 ? e : nbr_[slot - 1];
    sm[J::O_COEF + t] = el >= 0 ? T(u[(size_t)el * BS + r]) : T(0.0);
  }
  __syncthreads();

  // ---- phase A: base face states / fluxes and base volume states / fluxes
  const int nqf_items = 4 * NQF;
  for (int t = tid; t < nqf_items + NQV; t += blockDim.x) {
    if (t < nqf_items) {
      int lf = t / NQF, q = t - lf * NQF;
      int f = f_[lf];
      bool interior = nbr_[lf] >= 0;
      FacePtT<T> fp;
      load_face_pt(dm, NQF, f, q, interior, fp);
      fp_store(sm + J::O_FP + (lf * NQF + q) * J::NFP, fp);
      const int* fi = dm.face_info + 8 * f;
      const T* cL = sm + J::O_COEF + (side_[lf] == 0 ? 0 : 1 + lf) * BS;
      const T* cR = sm + J::O_COEF + (side_[lf] == 0 ? 1 + lf : 0) * BS;
      T* stL = sm + J::O_FST + ((lf * NQF + q) * 2 + 0) * NST;
      T* stR = sm + J::O_FST + ((lf * NQF + q) * 2 + 1) * NST;
      side_state<NB, NEQ, DDG>(cL, dm.tab_face + (size_t)((fi[2] * 2 + 0) * NQF + q) * NB * 6, fp.JiL, fp.HL, stL,
                               stL + NEQ, stL + 3 * NEQ);
      if (interior)
        side_state<NB, NEQ, DDG>(cR, dm.tab_face + (size_t)((fi[3] * 2 + fi[4]) * NQF + q) * NB * 6, fp.JiR, fp.HR,
                                 stR, stR + NEQ, stR + 3 * NEQ);
      const double* bval = interior ? nullptr : dm.bvals + ((size_t)bidx_[lf] * NQF + q) * NEQ;
      T out[NEQ], gq[4];
      face_flux_states<PDE, DDG, T>(pp, fp, interior, bct_[lf], bval, stL, stL + NEQ, stL + 3 * NEQ, stR, stR + NEQ,
                                    stR + 3 * NEQ, out, gq);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sm[J::O_FQB + (lf * NQF + q) * NEQ + k] = out[k];
      if (J::IC && ic)
#pragma unroll
        for (int k = 0; k < 4; ++k) sm[J::O_GQB + (lf * NQF + q) * 4 + k] = gq[k];
    } else {
      int q = t - nqf_items;
      int nq = dm.E * NQV;
      size_t kq = (size_t)e * NQV + q;
      T Ji[4] = {T(dm.vgeo[0 * nq + kq]), T(dm.vgeo[1 * nq + kq]), T(dm.vgeo[2 * nq + kq]), T(dm.vgeo[3 * nq + kq])};
      sm[J::O_WD + q] = T(dm.vgeo[4 * nq + kq]);
      const double* tb = dm.tab_vol + (size_t)q * NB * 3;
      const T* cf = sm + J::O_COEF;
      T uq[NEQ], gxi[NEQ][2];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) { uq[k] = T(0.0); gxi[k][0] = gxi[k][1] = T(0.0); }
      for (int i = 0; i < NB; ++i) {
        T phi = T(tb[i * 3]), d0 = T(tb[i * 3 + 1]), d1 = T(tb[i * 3 + 2]);
#pragma unroll
        for (int d = 0; d < 2; ++d)
          sm[J::O_GPHI + (q * NB + i) * 2 + d] = d0 * Ji[0 * 2 + d] + d1 * Ji[1 * 2 + d];
#pragma unroll
        for (int k = 0; k < NEQ; ++k) {
          T c = cf[i * NEQ + k];
          uq[k] += c * phi;
          gxi[k][0] += c * d0;
          gxi[k][1] += c * d1;
        }
      }
      T gx[2 * NEQ], F[2 * NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k)
#pragma unroll
        for (int d = 0; d < 2; ++d) gx[k * 2 + d] = gxi[k][0] * Ji[0 * 2 + d] + gxi[k][1] * Ji[1 * 2 + d];
      Phys<PDE>::flux(pp, uq, gx, F);
      T fro = T(0.0);
#pragma unroll
      for (int k = 0; k < 2 * NEQ; ++k) fro += F[k] * F[k];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sm[J::O_UQ + q * NEQ + k] = uq[k];
#pragma unroll
      for (int k = 0; k < 2 * NEQ; ++k) {
        sm[J::O_GQ + q * 2 * NEQ + k] = gx[k];
        sm[J::O_FB + q * 2 * NEQ + k] = F[k];
      }
      sm[J::O_EPSQ + q] = fmax(sqeps, sqrt(fro) * sqeps);
    }
  }
  __syncthreads();

  // ---- face perturbation sizes from the base face residual norms (one warp per face and side)
  {
    int warp = tid >> 5, lane = tid & 31;
    if (warp < 8) {
      int lf = warp >> 1, sd = warp & 1;  // sd: 0 = left element of the face, 1 = right
      bool interior = nbr_[lf] >= 0;
      T ss = T(0.0);
      if (sd == 0 || interior) {
        const int* fi = dm.face_info + 8 * f_[lf];
        int lfs = sd == 0 ? fi[2] : fi[3], os = sd == 0 ? 0 : fi[4];
        T sgn = sd == 0 ? T(1.0) : T(-1.0);
        for (int r = lane; r < BS; r += 32) {
          int i = r / NEQ, k = r - i * NEQ;
          T v = T(0.0);
#pragma unroll
          for (int q = 0; q < NQF; ++q) {
            const double* tf = dm.tab_face + ((size_t)((lfs * 2 + os) * NQF + q) * NB + i) * 6;
            v += sgn * T(tf[0]) * sm[J::O_FQB + (lf * NQF + q) * NEQ + k];
            if (J::IC && ic)
              v -= T(tf[1]) * sm[J::O_GQB + (lf * NQF + q) * 4 + sd * 2 + 0] +
                   T(tf[2]) * sm[J::O_GQB + (lf * NQF + q) * 4 + sd * 2 + 1];
          }
          ss += v * v;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, off);
      // two warps per face: combine through shared memory below
      if (lane == 0) sm[J::O_DFQ + warp] = sqrt(ss);  // scratch (overwritten in phase B)
    }
    __syncthreads();
    if (tid < 4) {
      int lf = tid;
      T nL = sm[J::O_DFQ + 2 * lf], nR = sm[J::O_DFQ + 2 * lf + 1];
      sm[J::O_EPSF + lf] = fmax(eps, fmax(nL, nR) * eps);
    }
    __syncthreads();
  }

  // ---- phase B: perturbed face fluxes (e's DOFs) and perturbed volume fluxes
  const int nfpert = BS * 4 * NQF;
  const int nvpert = NQV * NEQ * 3;
  for (int t = tid; t < nfpert + nvpert; t += blockDim.x) {
    if (t < nfpert) {
      int c = t / (4 * NQF), rem = t - c * 4 * NQF;
      int lf = rem / NQF, q = rem - lf * NQF;
      int j = c / NEQ, kc = c - j * NEQ;
      bool interior = nbr_[lf] >= 0;
      int se = side_[lf];
      FacePtT<T> fp;
      fp_load(sm + J::O_FP + (lf * NQF + q) * J::NFP, fp);
      T st[2][NST];
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int a = 0; a < NST; ++a) st[s][a] = sm[J::O_FST + ((lf * NQF + q) * 2 + s) * NST + a];
      T epsf = sm[J::O_EPSF + lf];
      const double* tfd = dm.tab_face + ((size_t)((lf * 2 + oe_[lf]) * NQF + q) * NB + j) * 6;
      T tf[6];
#pragma unroll
      for (int a = 0; a < 6; ++a) tf[a] = T(tfd[a]);
      T gphi[2], hphi[4];
      basis_phys<DDG>(tf, se ? fp.JiR : fp.JiL, se ? fp.HR : fp.HL, gphi, hphi);
      T* sv = st[se];
      sv[kc] += epsf * tf[0];
      sv[NEQ + kc * 2 + 0] += epsf * gphi[0];
      sv[NEQ + kc * 2 + 1] += epsf * gphi[1];
      if (DDG) {
#pragma unroll
        for (int a = 0; a < 4; ++a) sv[3 * NEQ + kc * 4 + a] += epsf * hphi[a];
      }
      const double* bval = interior ? nullptr : dm.bvals + ((size_t)bidx_[lf] * NQF + q) * NEQ;
      T out[NEQ], gq[4];
      face_flux_states<PDE, DDG, T>(pp, fp, interior, bct_[lf], bval, st[0], st[0] + NEQ, st[0] + 3 * NEQ, st[1],
                                    st[1] + NEQ, st[1] + 3 * NEQ, out, gq);
#pragma unroll
      for (int k = 0; k < NEQ; ++k)
        sm[J::O_DFQ + ((c * 4 + lf) * NQF + q) * NEQ + k] =
            (out[k] - sm[J::O_FQB + (lf * NQF + q) * NEQ + k]) / epsf;
      if (J::IC && ic)
#pragma unroll
        for (int k = 0; k < 4; ++k)
          sm[J::O_DGQ + ((c * 4 + lf) * NQF + q) * 4 + k] = (gq[k] - sm[J::O_GQB + (lf * NQF + q) * 4 + k]) / epsf;
    } else {
      int t2 = t - nfpert;
      int q = t2 / (NEQ * 3), pidx = t2 - q * NEQ * 3;
      T uq[NEQ], gx[2 * NEQ], F[2 * NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) uq[k] = sm[J::O_UQ + q * NEQ + k];
#pragma unroll
      for (int k = 0; k < 2 * NEQ; ++k) gx[k] = sm[J::O_GQ + q * 2 * NEQ + k];
      T epsq = sm[J::O_EPSQ + q];
      if (pidx < NEQ) uq[pidx] += epsq;
      else gx[pidx - NEQ] += epsq;
      Phys<PDE>::flux(pp, uq, gx, F);
      const T* Fb = sm + J::O_FB + q * 2 * NEQ;
      if (pidx < NEQ) {
        int je = pidx;
#pragma unroll
        for (int ie = 0; ie < NEQ; ++ie)
#pragma unroll
          for (int d = 0; d < 2; ++d)
            sm[J::O_DFDU + ((q * NEQ + ie) * 2 + d) * NEQ + je] = (F[ie * 2 + d] - Fb[ie * 2 + d]) / epsq;
      } else {
        int je = (pidx - NEQ) / 2, jd = (pidx - NEQ) & 1;
#pragma unroll
        for (int ie = 0; ie < NEQ; ++ie)
#pragma unroll
          for (int d = 0; d < 2; ++d)
            sm[J::O_DFDG + (((q * NEQ + ie) * 2 + d) * NEQ + je) * 2 + jd] = (F[ie * 2 + d] - Fb[ie * 2 + d]) / epsq;
      }
    }
  }
  __syncthreads();

  // ---- diagonal block: volume + the e-e coupling of the four faces
  T* Jd = vals + (size_t)dm.bsr_diag[e] * BS * BS;
  for (int t = tid; t < BS * BS; t += blockDim.x) {
    int r = t / BS, c = t - r * BS;
    int i = r / NEQ, ie = r - i * NEQ;
    int j = c / NEQ, je = c - j * NEQ;
    T acc = T(0.0);
    for (int q = 0; q < NQV; ++q) {
      const T* gi = sm + J::O_GPHI + (q * NB + i) * 2;
      const T* gj = sm + J::O_GPHI + (q * NB + j) * 2;
      T phij = T(dm.tab_vol[((size_t)q * NB + j) * 3]);
      T wd = sm[J::O_WD + q];
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        T term = sm[J::O_DFDU + ((q * NEQ + ie) * 2 + d) * NEQ + je] * phij;
        term += sm[J::O_DFDG + (((q * NEQ + ie) * 2 + d) * NEQ + je) * 2 + 0] * gj[0];
        term += sm[J::O_DFDG + (((q * NEQ + ie) * 2 + d) * NEQ + je) * 2 + 1] * gj[1];
        acc += term * gi[d] * wd;
      }
    }
#pragma unroll
    for (int lf = 0; lf < 4; ++lf) {
      T sgn = side_[lf] == 0 ? T(1.0) : T(-1.0);
      T s = T(0.0);
#pragma unroll
      for (int q = 0; q < NQF; ++q) {
        const double* tf = dm.tab_face + ((size_t)((lf * 2 + oe_[lf]) * NQF + q) * NB + i) * 6;
        s += sgn * T(tf[0]) * sm[J::O_DFQ + ((c * 4 + lf) * NQF + q) * NEQ + ie];
        if (J::IC && ic)
          s -= T(tf[1]) * sm[J::O_DGQ + ((c * 4 + lf) * NQF + q) * 4 + side_[lf] * 2 + 0] +
               T(tf[2]) * sm[J::O_DGQ + ((c * 4 + lf) * NQF + q) * 4 + side_[lf] * 2 + 1];
      }
      acc += s;
    }
    Jd[(size_t)r * BS + c] = acc;
  }

  // ---- neighbour blocks (n, e)
#pragma unroll 1
  for (int lf = 0; lf < 4; ++lf) {
    if (nbr_[lf] < 0) continue;
    int se = side_[lf], sn = 1 - se;
    int blk = dm.face_blk[f_[lf] * 4 + (se == 0 ? 2 : 1)];
    T* Jn = vals + (size_t)blk * BS * BS;
    T sgn = sn == 0 ? T(1.0) : T(-1.0);
    for (int t = tid; t < BS * BS; t += blockDim.x) {
      int r = t / BS, c = t - r * BS;
      int i = r / NEQ, ie = r - i * NEQ;
      T s = T(0.0);
#pragma unroll
      for (int q = 0; q < NQF; ++q) {
        const double* tf = dm.tab_face + ((size_t)((lfn_[lf] * 2 + on_[lf]) * NQF + q) * NB + i) * 6;
        s += sgn * T(tf[0]) * sm[J::O_DFQ + ((c * 4 + lf) * NQF + q) * NEQ + ie];
        if (J::IC && ic)
          s -= T(tf[1]) * sm[J::O_DGQ + ((c * 4 + lf) * NQF + q) * 4 + sn * 2 + 0] +
               T(tf[2]) * sm[J::O_DGQ + ((c * 4 + lf) * NQF + q) * 4 + sn * 2 + 1];
      }
      Jn[(size_t)r * BS + c] = s;
    }
  }
}

// ------------------------------------------------------------------ SpMV
// y = J x; one warp per block row, lanes over the rows of the block
template <int PDE, int P, int G, class T>
static cudaError_t jac_pg(const DeviceMesh& dm, const PhysParams& pp, const double* u, T* vals, double eps,
                          cudaStream_t s) {
  using J = JacCfg<PDE, P, G, T>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e1 = cudaFuncSetAttribute(jac_elem_kernel<PDE, P, G, true, T>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)J::SMEM);
    cudaError_t e2 = cudaFuncSetAttribute(jac_elem_kernel<PDE, P, G, false, T>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)J::SMEM);
    if (e1 != cudaSuccess) return e1;
    if (e2 != cudaSuccess) return e2;
    attr_set = true;
  }
  if (pp.beta1 != 0.0)
    jac_elem_kernel<PDE, P, G, true, T><<<dm.E, J::THREADS, J::SMEM, s>>>(dm, pp, u, vals, eps);
  else
    jac_elem_kernel<PDE, P, G, false, T><<<dm.E, J::THREADS, J::SMEM, s>>>(dm, pp, u, vals, eps);
  return cudaGetLastError();
}

template <class T>
static cudaError_t jac_dispatch(const DeviceMesh& dm, const PhysParams& pp, const double* u, T* vals, double eps,
                                cudaStream_t s) {
#define ICX_JAC_CASE(PDE, PP, GG) \
  if (pp.pde == PDE && dm.P == PP && dm.G == GG) return jac_pg<PDE, PP, GG, T>(dm, pp, u, vals, eps, s);
  ICX_JAC_CASE(0, 1, 1) ICX_JAC_CASE(0, 2, 1) ICX_JAC_CASE(0, 3, 1) ICX_JAC_CASE(0, 4, 1)
  ICX_JAC_CASE(0, 1, 2) ICX_JAC_CASE(0, 2, 2) ICX_JAC_CASE(0, 3, 2) ICX_JAC_CASE(0, 4, 2)
  ICX_JAC_CASE(1, 1, 1) ICX_JAC_CASE(1, 2, 1) ICX_JAC_CASE(1, 3, 1) ICX_JAC_CASE(1, 4, 1)
  ICX_JAC_CASE(1, 1, 2) ICX_JAC_CASE(1, 2, 2) ICX_JAC_CASE(1, 3, 2) ICX_JAC_CASE(1, 4, 2)
#undef ICX_JAC_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_jacobian_fd(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                               double* vals, double eps, cudaStream_t s) {
  cudaError_t e = launch_residual(dm, pp, u, res, s);
  if (e != cudaSuccess) return e;
  return jac_dispatch<double>(dm, pp, u, vals, eps, s);
}

// the FP64 residual and the FP32-quadrature Jacobian (T = float)
cudaError_t launch_jacobian_fd_f32(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                                   float* vals, cudaStream_t s) {
  cudaError_t e = launch_residual(dm, pp, u, res, s);
  if (e != cudaSuccess) return e;
  return jac_dispatch<float>(dm, pp, u, vals, std::sqrt((double)FLT_EPSILON), s);
}

cudaError_t launch_bsr_spmv(const DeviceMesh& dm, const double* vals, const double* x, double* y, cudaStream_t s) {
  int bs = dm.nb * dm.neq;
  RowSet rs{0, 0, -1, dm.E};
#define ICX_SPMV_CASE(B) \
  if (bs == B) return launch_block_rows<B, BR_ALL>(rs, dm.bsr_rowptr, dm.bsr_colidx, vals, x, nullptr, 1.0, y, s);
  ICX_BLOCK_SIZES(ICX_SPMV_CASE)
#undef ICX_SPMV_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_bsr_spmv_f32(const DeviceMesh& dm, const float* vals, const double* x, double* y, cudaStream_t s) {
  int bs = dm.nb * dm.neq;
  RowSet rs{0, 0, -1, dm.E};
#define ICX_SPMV32_CASE(B) \
  if (bs == B) return launch_block_rows<B, BR_ALL, float>(rs, dm.bsr_rowptr, dm.bsr_colidx, vals, x, nullptr, 1.0, y, s);
  ICX_BLOCK_SIZES(ICX_SPMV32_CASE)
#undef ICX_SPMV32_CASE
  return cudaErrorInvalidValue;
}

}  // namespace icx
