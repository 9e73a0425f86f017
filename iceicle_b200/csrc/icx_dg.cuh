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
template <bool WANT_H>
__device__ inline void basis_phys(const double* t, const double* Ji, const double* Hm, double* gx, double* hx) {
#pragma unroll
  for (int d = 0; d < 2; ++d) gx[d] = t[1] * Ji[0 * 2 + d] + t[2] * Ji[1 * 2 + d];
  if (WANT_H) {
    double r00 = t[3] - Hm[0] * gx[0] - Hm[3] * gx[1];
    double r01 = t[4] - Hm[1] * gx[0] - Hm[4] * gx[1];
    double r11 = t[5] - Hm[2] * gx[0] - Hm[5] * gx[1];
    double rhs[2][2] = {{r00, r01}, {r01, r11}};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        double s = 0.0;
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
// tab: [NB][6] = phi, dphi/dxi0, dphi/dxi1, h00, h01, h11.
template <int NB, int NEQ, bool WANT_H>
__device__ inline void side_state(const double* __restrict__ ue, const double* __restrict__ tab, const double* Ji,
                                  const double* Hm, double* u, double* gx, double* hx) {
  double gxi[NEQ][2], hxi[NEQ][3];
#pragma unroll
  for (int eq = 0; eq < NEQ; ++eq) {
    u[eq] = 0.0;
    gxi[eq][0] = gxi[eq][1] = 0.0;
    hxi[eq][0] = hxi[eq][1] = hxi[eq][2] = 0.0;
  }
#pragma unroll 4
  for (int i = 0; i < NB; ++i) {
    const double* t = tab + i * 6;
    double phi = t[0], d0 = t[1], d1 = t[2];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) {
      double c = ue[i * NEQ + eq];
      u[eq] += c * phi;
      gxi[eq][0] += c * d0;
      gxi[eq][1] += c * d1;
      if (WANT_H) {
        hxi[eq][0] += c * t[3];
        hxi[eq][1] += c * t[4];
        hxi[eq][2] += c * t[5];
      }
    }
  }
#pragma unroll
  for (int eq = 0; eq < NEQ; ++eq) {
    double tt[6] = {0.0, gxi[eq][0], gxi[eq][1], hxi[eq][0], hxi[eq][1], hxi[eq][2]};
    basis_phys<WANT_H>(tt, Ji, Hm, gx + eq * 2, hx + eq * 4);
  }
}

// geometry of one face quadrature point (both sides)
struct FacePt {
  double n[2], wsq, h;
  double JiL[4], HL[6], JiR[4], HR[6];
};

__device__ inline void load_face_pt(const DeviceMesh& dm, int nqf, int f, int q, bool interior, FacePt& p) {
  int nfq = dm.F * nqf, k = f * nqf + q;
  const double* g = dm.fgeo;
  p.n[0] = g[FG_N0 * nfq + k];
  p.n[1] = g[FG_N1 * nfq + k];
  p.wsq = g[FG_WSQ * nfq + k];
  p.h = g[FG_H * nfq + k];
#pragma unroll
  for (int a = 0; a < 4; ++a) p.JiL[a] = g[(FG_JIL + a) * nfq + k];
#pragma unroll
  for (int a = 0; a < 6; ++a) p.HL[a] = g[(FG_HL + a) * nfq + k];
  if (interior) {
#pragma unroll
    for (int a = 0; a < 4; ++a) p.JiR[a] = g[(FG_JIR + a) * nfq + k];
#pragma unroll
    for (int a = 0; a < 6; ++a) p.HR[a] = g[(FG_HR + a) * nfq + k];
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
template <int PDE>
__device__ inline bool face_exterior(const PhysParams& pp, const FacePt& fp, int bct, const double* bval,
                                     const double* uL, double* ud) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  if (bct == ICX_BC_DIRICHLET || (bct == ICX_BC_SPACETIME_PAST && pp.st_connected)) {
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) ud[eq] = bval[eq];
    return true;
  }
  if (Phys<PDE>::has_pde_bcs && bct >= ICX_BC_RIEMANN && bct <= ICX_BC_WALL_GENERAL) {
    Phys<PDE>::apply_bc(pp, uL, fp.n, bct, bval, ud);
    return true;
  }
  return false;
}

// convective part (zero where the face has none) and the interface-correction coefficients
template <int PDE, bool DDG>
__device__ inline void face_conv_part(const PhysParams& pp, const FacePt& fp, bool interior, int bct,
                                      const double* bval, const double* uL, const double* uR, double* fadv,
                                      double* gq) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  const double* n = fp.n;
  const double wsq = fp.wsq;
  const bool ic = Phys<PDE>::has_ic && pp.sigma_ic != 0.0;
  double ud[NEQ];
  if (interior) {
    Phys<PDE>::conv_sel(pp, uL, uR, n, fadv);
    if (ic) {
      // resL, resR -= sum_s (sigma mu n_s [u] w sqrt(g) / 2) dphi/dx_s   (conservation_law.hpp:580-610)
      double cs[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) cs[s] = 0.5 * pp.sigma_ic * pp.mu * n[s] * (uR[0] - uL[0]) * wsq;
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        gq[0 * 2 + kk] = cs[0] * fp.JiL[kk * 2 + 0] + cs[1] * fp.JiL[kk * 2 + 1];
        gq[1 * 2 + kk] = cs[0] * fp.JiR[kk * 2 + 0] + cs[1] * fp.JiR[kk * 2 + 1];
      }
    }
  } else if (face_exterior<PDE>(pp, fp, bct, bval, uL, ud)) {
    // a connected SPACETIME_PAST face takes the past slab's trace as exterior
    // state; on a slab interface at constant t the diffusive normal flux
    // vanishes (no diffusion along t), leaving the time-upwind flux. The
    // PDE-level kinds (walls, characteristic) form the exterior state from
    // the interior one and then take the same DDG boundary flux as a
    // Dirichlet face with one-sided gradients (conservation_law.hpp:1043-1130)
    Phys<PDE>::conv_sel(pp, uL, ud, n, fadv);
    if (ic) {
      // resL -= sum_s sigma mu n_s [u] w sqrt(g) dphi/dx_s   (conservation_law.hpp:735-760)
      double cs[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) cs[s] = pp.sigma_ic * pp.mu * n[s] * (ud[0] - uL[0]) * wsq;
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        gq[0 * 2 + kk] = cs[0] * fp.JiL[kk * 2 + 0] + cs[1] * fp.JiL[kk * 2 + 1];
        gq[1 * 2 + kk] = 0.0;
      }
    }
  } else if (bct == ICX_BC_EXTRAPOLATION || bct == ICX_BC_SPACETIME_FUTURE) {
    Phys<PDE>::conv_sel(pp, uL, uL, n, fadv);
    if (ic) gq[0] = gq[1] = gq[2] = gq[3] = 0.0;
  } else {
    // Neumann faces have no convective part; boundary kinds the PDE does not
    // implement contribute nothing
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) fadv[eq] = 0.0;
    if (ic) gq[0] = gq[1] = gq[2] = gq[3] = 0.0;
  }
}

// viscous part (zero where the face has none)
template <int PDE, bool DDG>
__device__ inline void face_visc_part(const PhysParams& pp, const FacePt& fp, bool interior, int bct,
                                      const double* bval, const double* uL, const double* gL, const double* hL,
                                      const double* uR, const double* gR, const double* hR, double* fvis) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  const double* n = fp.n;
  const double h = fp.h;
  double ud[NEQ];
  if (interior) {
    double gddg[2 * NEQ], uavg[NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) {
      double jump = uR[eq] - uL[eq];
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        double v = pp.beta0 * jump / h * n[d] + 0.5 * (gL[eq * 2 + d] + gR[eq * 2 + d]);
        if (DDG) {
          double ht = (hR[eq * 4 + 0 * 2 + d] - hL[eq * 4 + 0 * 2 + d]) * n[0] +
                      (hR[eq * 4 + 1 * 2 + d] - hL[eq * 4 + 1 * 2 + d]) * n[1];
          v += pp.beta1 * h * ht;
        }
        gddg[eq * 2 + d] = v;
      }
      uavg[eq] = 0.5 * (uL[eq] + uR[eq]);
    }
    Phys<PDE>::diff(pp, uavg, gddg, n, fvis);
  } else if (face_exterior<PDE>(pp, fp, bct, bval, uL, ud)) {
    double gddg[2 * NEQ], uavg[NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) {
#pragma unroll
      for (int d = 0; d < 2; ++d) gddg[eq * 2 + d] = pp.beta0 * (ud[eq] - uL[eq]) / h * n[d] + gL[eq * 2 + d];
      uavg[eq] = 0.5 * (uL[eq] + ud[eq]);
    }
    Phys<PDE>::diff(pp, uavg, gddg, n, fvis);
  } else if (bct == ICX_BC_NEUMANN) {
    double gn[NEQ];
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) gn[eq] = bval[eq];
    Phys<PDE>::neumann(pp, gn, fvis);
  } else if (bct == ICX_BC_EXTRAPOLATION || bct == ICX_BC_SPACETIME_FUTURE) {
    Phys<PDE>::diff(pp, uL, gL, n, fvis);
  } else {
#pragma unroll
    for (int eq = 0; eq < NEQ; ++eq) fvis[eq] = 0.0;
  }
}

template <int PDE>
__device__ inline void face_combine(const FacePt& fp, const double* fvis, const double* fadv, double* out) {
#pragma unroll
  for (int eq = 0; eq < Phys<PDE>::NEQ; ++eq) out[eq] = fvis[eq] * fp.wsq - fadv[eq] * fp.wsq;
}

template <int PDE, bool DDG>
__device__ inline void face_flux_states(const PhysParams& pp, const FacePt& fp, bool interior, int bct,
                                        const double* bval, const double* uL, const double* gL, const double* hL,
                                        const double* uR, const double* gR, const double* hR, double* out,
                                        double* gq) {
  constexpr int NEQ = Phys<PDE>::NEQ;
  double fadv[NEQ], fvis[NEQ];
  face_conv_part<PDE, DDG>(pp, fp, interior, bct, bval, uL, uR, fadv, gq);
  face_visc_part<PDE, DDG>(pp, fp, interior, bct, bval, uL, gL, hL, uR, gR, hR, fvis);
  face_combine<PDE>(fp, fvis, fadv, out);
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
