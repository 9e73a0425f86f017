// Device building blocks shared by the residual and the FD-Jacobian kernels:
// compile-time sizes, the solution state on one side of a face point, and the
// numerical flux at a face point given both sides' states
// (trace_integral / boundaryIntegral, conservation_law.hpp:434-1176).
#pragma once
#include <cfloat>

#include "icx_internal.h"
#include "icx_physics.cuh"

namespace icx {

template <int PDE, int P, int G>
struct Cfg {
  static constexpr int NEQ = Phys<PDE>::NEQ;
  static constexpr int NB = (P + 1) * (P + 1);
  static constexpr int BS = NB * NEQ;
  static constexpr int NQ1 = G + P;
  static constexpr int NQV = NQ1 * NQ1;
  static constexpr int NQF = NQ1;
  static constexpr int NG = (G + 1) * (G + 1);
};

// physical parameters of element e: in a batch of independent Burgers
// problems each element carries its problem's coefficients (mu, a, b)
template <int PDE>
__device__ inline PhysParams elem_params(const DeviceMesh& dm, const PhysParams& pp, int e) {
  PhysParams q = pp;
  if (PDE == ICX_PDE_BURGERS && dm.el_par) {
    const double* v = dm.el_par + 5 * (size_t)e;
    q.mu = v[0];
    q.mu_t = v[0];  // batches hold plain (not spacetime) Burgers parts
    q.a[0] = v[1];
    q.a[1] = v[2];
    q.b[0] = v[3];
    q.b[1] = v[4];
  }
  return q;
}

// physical gradient (and Hessian) of one basis function from its reference
// derivatives t = [phi, d0, d1, h00, h01, h11]:
//   dx = Ji^T dxi,  Hx = Ji^T (Hxi - sum_m Hm_m dx_m) Ji   (finite_element.hpp:220-398)
template <bool WANT_H, class T>
__device__ inline void basis_phys(const T* t, const T* Ji, const T* Hm, T* gx, T* hx) {
#pragma unroll
  for (int d = 0; d < 2; ++d) gx[d] = t[1] * Ji[0 * 2 + d] + t[2] * Ji[1 * 2 + d];
  if (WANT_H) {
    T r00 = t[3] - Hm[0] * gx[0] - Hm[3] * gx[1];
    T r01 = t[4] - Hm[1] * gx[0] - Hm[4] * gx[1];
    T r11 = t[5] - Hm[2] * gx[0] - Hm[5] * gx[1];
    T rhs[2][2] = {{r00, r01}, {r01, r11}};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        T s = T(0.0);
#pragma unroll
        for (int l = 0; l < 2; ++l)
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) s += Ji[l * 2 + a] * rhs[l][kk] * Ji[kk * 2 + b];
        hx[a * 2 + b] = s;
      }
  }
}

// value, physical gradient [NEQ][2] and (if WANT_H) physical Hessian
// [NEQ][2][2] of the solution on one side of a face point.
// tab: [NB][6] = phi, dphi/dxi0, dphi/dxi1, h00, h01, h11 (FP64 tables; an
// FP32 evaluation rounds each entry once as it reads it).
template <int NB, int NEQ, bool WANT_H, class T>
__device__ inline void side_state(const T* __restrict__ ue, const double* __restrict__ tab, const T* Ji,
                                  const T* Hm, T* u, T* gx, T* hx) {
  T gxi[NEQ][2], hxi[NEQ][3];
#pragma unroll
  for (int eq = 0; eq < NEQ; ++eq) {
    u[eq] = T(0.0);
    gxi[eq][0] = gxi[eq][1] = T(0.0);
    hxi[eq][0] = hxi[eq][1] = hxi[eq][2] = T(0.0);
  }
#pragma unroll 4
  for (int i = 0; i < NB; ++i) {
    const double* t = tab + i * 6;
    T phi = T(t[0]), d0 = T(t[1]), d1 = T(t[2]);
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) {
      T c = ue[i * NEQ + eq];
      u[eq] += c * phi;
      gxi[eq][0] += c * d0;
      gxi[eq][1] += c * d1;
      if (WANT_H) {
        hxi[eq][0] += c * T(t[3]);
        hxi[eq][1] += c * T(t[4]);
        hxi[eq][2] += c * T(t[5]);
      }
    }
  }
#pragma unroll
  for (int eq = 0; eq < NEQ; ++eq) {
    T tt[6] = {T(0.0), gxi[eq][0], gxi[eq][1], hxi[eq][0], hxi[eq][1], hxi[eq][2]};
    basis_phys<WANT_H>(tt, Ji, Hm, gx + eq * 2, hx + eq * 4);
  }
}

// geometry of one face quadrature point (both sides); the FP32 form holds
// the FP64 metrics rounded once
template <class T>
struct FacePtT {
  T n[2], wsq, h;
  T JiL[4], HL[6], JiR[4], HR[6];
};
using FacePt = FacePtT<double>;

template <class T>
__device__ inline void load_face_pt(const DeviceMesh& dm, int nqf, int f, int q, bool interior, FacePtT<T>& p) {
  int nfq = dm.F * nqf, k = f * nqf + q;
  const double* g = dm.fgeo;
  p.n[0] = T(g[FG_N0 * nfq + k]);
  p.n[1] = T(g[FG_N1 * nfq + k]);
  p.wsq = T(g[FG_WSQ * nfq + k]);
  p.h = T(g[FG_H * nfq + k]);
#pragma unroll
  for (int a = 0; a < 4; ++a) p.JiL[a] = T(g[(FG_JIL + a) * nfq + k]);
#pragma unroll
  for (int a = 0; a < 6; ++a) p.HL[a] = T(g[(FG_HL + a) * nfq + k]);
  if (interior) {
#pragma unroll
    for (int a = 0; a < 4; ++a) p.JiR[a] = T(g[(FG_JIR + a) * nfq + k]);
#pragma unroll
    for (int a = 0; a < 6; ++a) p.HR[a] = T(g[(FG_HR + a) * nfq + k]);
  }
}

// numerical flux at a face point from both sides' states, in two parts that
// the face kernel may evaluate on two threads: the convective part fadv
// (face_conv_part, also the interface-correction coefficients gq) and the
// viscous part fvis (face_visc_part); face_flux_states runs both.
// out[NEQ] = (f_visc - f_adv) * w * sqrt(g); with the interface correction
// active, gq[4] = the pulled-back coefficients of dphi/dxi for the left
// (gq[0..1]) and right (gq[2..3]) test functions.
// bval: Dirichlet state or Neumann data at this boundary point.

// the exterior state of a boundary point whose flux uses one: Dirichlet data,
// a connected past slab, or a PDE-level boundary; false for the other kinds
template <int PDE, class T>
__device__ inline bool face_exterior(const PhysParams& pp, const FacePtT<T>& fp, int bct, const double* bval,
                                     const T* uL, T* ud) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  if (bct == ICX_BC_DIRICHLET || (bct == ICX_BC_SPACETIME_PAST && pp.st_connected)) {
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) ud[eq] = T(bval[eq]);
    return true;
  }
  if (Phys<PDE>::has_pde_bcs && bct >= ICX_BC_RIEMANN && bct <= ICX_BC_WALL_GENERAL) {
    Phys<PDE>::apply_bc(pp, uL, fp.n, bct, bval, ud);
    return true;
  }
  return false;
}

// convective part (zero where the face has none) and the interface-correction coefficients
template <int PDE, bool DDG, class T>
__device__ inline void face_conv_part(const PhysParams& pp, const FacePtT<T>& fp, bool interior, int bct,
                                      const double* bval, const T* uL, const T* uR, T* fadv, T* gq) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  const T* n = fp.n;
  const T wsq = fp.wsq;
  const bool ic = Phys<PDE>::has_ic && pp.sigma_ic != 0.0;
  T ud[NEQ];
  if (interior) {
    Phys<PDE>::conv_sel(pp, uL, uR, n, fadv);
    if (ic) {
      // resL, resR -= sum_s (sigma mu n_s [u] w sqrt(g) / 2) dphi/dx_s   (conservation_law.hpp:580-610)
      T cs[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) cs[s] = T(0.5) * T(pp.sigma_ic) * T(pp.mu) * n[s] * (uR[0] - uL[0]) * wsq;
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        gq[0 * 2 + kk] = cs[0] * fp.JiL[kk * 2 + 0] + cs[1] * fp.JiL[kk * 2 + 1];
        gq[1 * 2 + kk] = cs[0] * fp.JiR[kk * 2 + 0] + cs[1] * fp.JiR[kk * 2 + 1];
      }
    }
  } else if (face_exterior<PDE, T>(pp, fp, bct, bval, uL, ud)) {
    // a connected SPACETIME_PAST face takes the past slab's trace as exterior
    // state; on a slab interface at constant t the diffusive normal flux
    // vanishes (no diffusion along t), leaving the time-upwind flux. The
    // PDE-level kinds (walls, characteristic) form the exterior state from
    // the interior one and then take the same DDG boundary flux as a
    // Dirichlet face with one-sided gradients (conservation_law.hpp:1043-1130)
    Phys<PDE>::conv_sel(pp, uL, ud, n, fadv);
    if (ic) {
      // resL -= sum_s sigma mu n_s [u] w sqrt(g) dphi/dx_s   (conservation_law.hpp:735-760)
      T cs[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) cs[s] = T(pp.sigma_ic) * T(pp.mu) * n[s] * (ud[0] - uL[0]) * wsq;
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        gq[0 * 2 + kk] = cs[0] * fp.JiL[kk * 2 + 0] + cs[1] * fp.JiL[kk * 2 + 1];
        gq[1 * 2 + kk] = T(0.0);
      }
    }
  } else if (bct == ICX_BC_EXTRAPOLATION || bct == ICX_BC_SPACETIME_FUTURE) {
    Phys<PDE>::conv_sel(pp, uL, uL, n, fadv);
    if (ic) gq[0] = gq[1] = gq[2] = gq[3] = T(0.0);
  } else {
    // Neumann faces have no convective part; boundary kinds the PDE does not
    // implement contribute nothing
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) fadv[eq] = T(0.0);
    if (ic) gq[0] = gq[1] = gq[2] = gq[3] = T(0.0);
  }
}

// viscous part (zero where the face has none)
template <int PDE, bool DDG, class T>
__device__ inline void face_visc_part(const PhysParams& pp, const FacePtT<T>& fp, bool interior, int bct,
                                      const double* bval, const T* uL, const T* gL, const T* hL, const T* uR,
                                      const T* gR, const T* hR, T* fvis) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  const T* n = fp.n;
  const T h = fp.h;
  T ud[NEQ];
  if (interior) {
    T gddg[2 * NEQ], uavg[NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) {
      T jump = uR[eq] - uL[eq];
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        T v = T(pp.beta0) * jump / h * n[d] + T(0.5) * (gL[eq * 2 + d] + gR[eq * 2 + d]);
        if (DDG) {
          T ht = (hR[eq * 4 + 0 * 2 + d] - hL[eq * 4 + 0 * 2 + d]) * n[0] +
                 (hR[eq * 4 + 1 * 2 + d] - hL[eq * 4 + 1 * 2 + d]) * n[1];
          v += T(pp.beta1) * h * ht;
        }
        gddg[eq * 2 + d] = v;
      }
      uavg[eq] = T(0.5) * (uL[eq] + uR[eq]);
    }
    Phys<PDE>::diff(pp, uavg, gddg, n, fvis);
  } else if (face_exterior<PDE, T>(pp, fp, bct, bval, uL, ud)) {
    T gddg[2 * NEQ], uavg[NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) {
#pragma unroll
      for (int d = 0; d < 2; ++d) gddg[eq * 2 + d] = T(pp.beta0) * (ud[eq] - uL[eq]) / h * n[d] + gL[eq * 2 + d];
      uavg[eq] = T(0.5) * (uL[eq] + ud[eq]);
    }
    Phys<PDE>::diff(pp, uavg, gddg, n, fvis);
  } else if (bct == ICX_BC_NEUMANN) {
    T gn[NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) gn[eq] = T(bval[eq]);
    Phys<PDE>::neumann(pp, gn, fvis);
  } else if (bct == ICX_BC_EXTRAPOLATION || bct == ICX_BC_SPACETIME_FUTURE) {
    Phys<PDE>::diff(pp, uL, gL, n, fvis);
  } else {
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) fvis[eq] = T(0.0);
  }
}

template <int PDE, class T>
__device__ inline void face_combine(const FacePtT<T>& fp, const T* fvis, const T* fadv, T* out) {
#pragma unroll
  for (int eq = 0; eq < Phys<PDE>::NEQ; ++eq) out[eq] = fvis[eq] * fp.wsq - fadv[eq] * fp.wsq;
}

template <int PDE, bool DDG, class T>
__device__ inline void face_flux_states(const PhysParams& pp, const FacePtT<T>& fp, bool interior, int bct,
                                        const double* bval, const T* uL, const T* gL, const T* hL, const T* uR,
                                        const T* gR, const T* hR, T* out, T* gq) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  T fadv[NEQ], fvis[NEQ];
  face_conv_part<PDE, DDG, T>(pp, fp, interior, bct, bval, uL, uR, fadv, gq);
  face_visc_part<PDE, DDG, T>(pp, fp, interior, bct, bval, uL, gL, hL, uR, gR, hR, fvis);
  face_combine<PDE, T>(fp, fvis, fadv, out);
}

// numerical flux at face point (f, q) from the coefficient tiles of both sides
template <int PDE, int P, int G, bool DDG>
__device__ inline void face_point_flux(const DeviceMesh& dm, const PhysParams& pp, int f, int q,
                                       const double* __restrict__ uL_coef, const double* __restrict__ uR_coef,
                                       double* out, double* gq) {
  using C = Cfg<PDE, P, G>;
  constexpr int NEQ = C::NEQ, NB = C::NB, NQF = C::NQF;
  const int* fi = dm.face_info + 8 * f;
  int R = fi[1], fnl = fi[2], fnr = fi[3], orient = fi[4], bct = fi[5], bidx = fi[7];
  bool interior = R >= 0;
  FacePt fp;
  load_face_pt(dm, NQF, f, q, interior, fp);
  double uL[NEQ], gL[2 * NEQ], hL[4 * NEQ];
  double uR[NEQ], gR[2 * NEQ], hR[4 * NEQ];
  side_state<NB, NEQ, DDG>(uL_coef, dm.tab_face + (size_t)((fnl * 2 + 0) * NQF + q) * NB * 6, fp.JiL, fp.HL, uL, gL,
                           hL);
  if (interior)
    side_state<NB, NEQ, DDG>(uR_coef, dm.tab_face + (size_t)((fnr * 2 + orient) * NQF + q) * NB * 6, fp.JiR, fp.HR,
                             uR, gR, hR);
  const double* bval = interior ? nullptr : dm.bvals + ((size_t)bidx * NQF + q) * NEQ;
  face_flux_states<PDE, DDG>(pp, fp, interior, bct, bval, uL, gL, hL, uR, gR, hR, out, gq);
}

}  // namespace icx
