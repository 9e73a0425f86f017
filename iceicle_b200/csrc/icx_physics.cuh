// Pointwise physics as device functions: Burgers (physical flux, upwind
// numerical flux, diffusive normal flux) and compressible Navier-Stokes in
// conservative variables with unit reference parameters (physical flux, Van
// Leer flux splitting, viscous normal flux). Formulas follow, term by term:
//   burgers.hpp:41-250, navier_stokes.hpp:321-449 (EoS), 554-587 (gradients),
//   700-746 (stress, heat flux), 776-864 (Van Leer), 916-973 (flux),
//   1241-1289 (diffusion flux)  [src/FiniteElement/include/iceicle/disc/].
#pragma once
#include "icx_internal.h"

namespace icx {

template <int PDE> struct Phys;

// Every function is a template on the scalar type T of the states and
// fluxes: double for the residual and the FP64 Jacobian, float for the FP32
// flux quadrature of the mixed-precision Jacobian. Parameters are held in
// double (PhysParams) and rounded to T where they enter.

// ------------------------------------------------------------------ Burgers
template <> struct Phys<ICX_PDE_BURGERS> {
  static constexpr int NEQ = 1;

  // F_d = (a_d + b_d u / 2) u - mu_d du/dx_d, mu_0 = mu, mu_1 = mu_t (mu, or 0
  // in spacetime form where the second coordinate is time: a_1 = 1, b_1 = 0
  // give F_t = u, burgers.hpp:261-340)
  template <class T>
  __device__ static inline void flux(const PhysParams& pp, const T* u, const T* g, T* F) {
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      T lam = T(pp.a[d]) + T(0.5) * T(pp.b[d]) * u[0];
      F[d] = lam * u[0] - T(d == 0 ? pp.mu : pp.mu_t) * g[d];
    }
  }
  // upwinding on the averaged wavespeed P = n.(a + b uavg / 2)
  template <class T>
  __device__ static inline void conv(const PhysParams& pp, const T* uL, const T* uR, const T* n, T* f) {
    T uavg = T(0.5) * (uL[0] + uR[0]);
    T P = T(0.0);
#pragma unroll
    for (int d = 0; d < 2; ++d) P += n[d] * (T(pp.a[d]) + T(0.5) * T(pp.b[d]) * uavg);
    T uup = (P > T(0)) ? uL[0] : uR[0];
    T fa = T(0.0);
#pragma unroll
    for (int d = 0; d < 2; ++d) fa += n[d] * (T(pp.a[d]) + T(0.5) * T(pp.b[d]) * uup);
    f[0] = fa * uup;
  }
  template <class T>
  __device__ static inline void diff(const PhysParams& pp, const T* u, const T* g, const T* n, T* f) {
    f[0] = T(pp.mu) * g[0] * n[0] + T(pp.mu_t) * g[1] * n[1];
  }
  template <class T>
  __device__ static inline void neumann(const PhysParams& pp, const T* gn, T* f) { f[0] = T(pp.mu) * gn[0]; }
  static constexpr bool has_ic = true;  // homogeneity tensor G = mu * I
  template <class T>
  __device__ static inline void conv_sel(const PhysParams& pp, const T* uL, const T* uR, const T* n, T* f) {
    conv(pp, uL, uR, n, f);
  }
  // the Burgers fluxes implement no PDE-level boundaries: those faces contribute nothing
  static constexpr bool has_pde_bcs = false;
  template <class T>
  __device__ static inline void apply_bc(const PhysParams&, const T* uL, const T*, int, const double*, T* uR) {
    uR[0] = uL[0];
  }
};

// ------------------------------------------------------------ Navier-Stokes
template <class T>
struct NSState {
  T rho, mom0, mom1, rhoE, v0, v1, vv, p, c, E, inv_rho;
};

constexpr double NS_RGAS = 287.052874;

// Quotients by the density are taken as products with one reciprocal per
// state (a last-bit difference from dividing each time).
template <class T>
__device__ static inline NSState<T> ns_state(const PhysParams& pp, const T* u) {
  NSState<T> s;
  T gamma = T(pp.gamma);
  s.rho = fmax(T(1e-14), u[0]);
  s.inv_rho = T(1.0) / s.rho;
  s.mom0 = u[1];
  s.mom1 = u[2];
  s.v0 = u[1] * s.inv_rho;
  s.v1 = u[2] * s.inv_rho;
  s.vv = s.v0 * s.v0 + s.v1 * s.v1;
  s.rhoE = u[3];
  s.E = s.rhoE * s.inv_rho;
  T e = s.E - T(0.5) * s.vv;
  s.p = fmax(T(1e-12), (gamma - T(1)) * s.rho * e);
  s.c = sqrt(gamma * s.p * s.inv_rho);
  return s;
}

template <> struct Phys<ICX_PDE_NAVIER_STOKES> {
  static constexpr int NEQ = 4;

  // the viscosity at the state's temperature T = p / rho * gamma / (gamma - 1) / cp
  // (constant_viscosity, or DimensionlessSutherlands, navier_stokes.hpp:226-287)
  template <class T>
  __device__ static inline T viscosity(const PhysParams& pp, const NSState<T>& s) {
    if (pp.ns_visc != 1) return T(pp.ns_mu);
    const T gam = T(pp.gamma);
    const T cp = gam / (gam - T(1)) * T(pp.Rgas);
    const T temp = s.p * s.inv_rho * gam / (gam - T(1)) / cp;
    const T t0 = T(pp.suth[1]), ts = T(pp.suth[2]);
    return T(pp.suth[0]) * pow(temp / t0, T(1.5)) * (t0 + ts) / (temp + ts);
  }

  // velocity gradients gv[i][j] and total energy gradient gE[j]; shear
  // stress; mgp = mu gamma / Pr of the heat flux
  template <class T>
  __device__ static inline void viscous(const PhysParams& pp, const NSState<T>& s, const T* g, T tau[2][2],
                                        T gv[2][2], T gE[2], T& mgp) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) gv[i][j] = (g[2 * (1 + i) + j] - (i == 0 ? s.v0 : s.v1) * g[j]) * s.inv_rho;
#pragma unroll
    for (int j = 0; j < 2; ++j) gE[j] = (g[6 + j] - s.E * g[j]) * s.inv_rho;
    T mu = viscosity(pp, s);
    mgp = pp.ns_visc == 1 ? mu * T(pp.gamma) / T(pp.Pr) : T(pp.mu_gamma_pr);
    T div = gv[0][0] + gv[1][1];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) tau[i][j] = mu * (gv[i][j] + gv[j][i]);
    tau[0][0] -= T(2.0 / 3.0) * mu * div;
    tau[1][1] -= T(2.0 / 3.0) * mu * div;
  }

  template <class T>
  __device__ static inline void flux(const PhysParams& pp, const T* u, const T* g, T* F) {
    NSState<T> s = ns_state(pp, u);
    T vel[2] = {s.v0, s.v1}, mom[2] = {s.mom0, s.mom1};
    // F[eq*2 + j]
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      F[0 * 2 + j] = mom[j];
#pragma unroll
      for (int i = 0; i < 2; ++i) F[(1 + i) * 2 + j] = mom[i] * vel[j];
      F[(1 + j) * 2 + j] += s.p;
      F[3 * 2 + j] = vel[j] * (s.rhoE + s.p);
    }
    T tau[2][2], gv[2][2], gE[2], mgp;
    viscous(pp, s, g, tau, gv, gE, mgp);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      T q = gE[j];
      q -= vel[0] * gv[0][j];
      q -= vel[1] * gv[1][j];
      q *= mgp;
      T ef = q;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        F[(1 + i) * 2 + j] -= tau[i][j];
        ef += vel[i] * tau[i][j];
      }
      F[3 * 2 + j] -= ef;
    }
  }

  // Van Leer flux vector splitting on the normal Mach number
  template <class T>
  __device__ static inline void conv(const PhysParams& pp, const T* uL, const T* uR, const T* n, T* f) {
    NSState<T> L = ns_state(pp, uL), R = ns_state(pp, uR);
    T gam = T(pp.gamma);
    T vnL = L.v0 * n[0] + L.v1 * n[1];
    T vnR = R.v0 * n[0] + R.v1 * n[1];
    T mL = vnL / L.c, mR = vnR / R.c;
    const T inv_gam = T(pp.inv_gamma), inv_g21 = T(pp.inv_2gam2m1);
    if (mL > T(1)) {
      f[0] = L.rho * vnL;
      f[1] = L.mom0 * vnL + L.p * n[0];
      f[2] = L.mom1 * vnL + L.p * n[1];
      f[3] = vnL * (L.rhoE + L.p);
    } else if (mL < T(-1)) {
      f[0] = f[1] = f[2] = f[3] = T(0.0);
    } else {
      T fmL = L.rho * L.c * (mL + T(1)) * (mL + T(1)) / T(4.0);
      f[0] = fmL;
      f[1] = fmL * (L.v0 + n[0] * (-vnL + T(2) * L.c) * inv_gam);
      f[2] = fmL * (L.v1 + n[1] * (-vnL + T(2) * L.c) * inv_gam);
      T t = (gam - T(1)) * vnL + T(2) * L.c;
      f[3] = fmL * ((L.vv - vnL * vnL) / T(2) + t * t * inv_g21);
    }
    if (mR < T(-1)) {
      f[0] += R.rho * vnR;
      f[1] += R.mom0 * vnR + R.p * n[0];
      f[2] += R.mom1 * vnR + R.p * n[1];
      f[3] += vnR * (R.rhoE + R.p);
    } else if (mR <= T(1)) {
      T fmR = -R.rho * R.c * (mR - T(1)) * (mR - T(1)) / T(4.0);
      f[0] += fmR;
      f[1] += fmR * (R.v0 + n[0] * (-vnR - T(2) * R.c) * inv_gam);
      f[2] += fmR * (R.v1 + n[1] * (-vnR - T(2) * R.c) * inv_gam);
      T t = (gam - T(1)) * vnR - T(2) * R.c;
      f[3] += fmR * ((R.vv - vnR * vnR) / T(2) + t * t * inv_g21);
    }
  }

  // Roe's approximate Riemann solver (P. L. Roe, J. Comput. Phys. 43, 1981):
  // F = (F(uL).n + F(uR).n) / 2 - sum_k |lambda_k| alpha_k r_k / 2 over the
  // acoustic, entropy and shear waves of the Roe-averaged state, with
  // Harten's entropy fix on the acoustic eigenvalues
  // (|l| < d: (l^2 + d^2) / (2 d), d = 0.1 c~). Unit reference parameters
  // (Eu = e_coeff = 1), so the ideal-gas relations take their usual form.
  template <class T>
  __device__ static inline void roe(const PhysParams& pp, const T* uL, const T* uR, const T* n, T* f) {
    NSState<T> L = ns_state(pp, uL), R = ns_state(pp, uR);
    const T gam = T(pp.gamma);
    const T vnL = L.v0 * n[0] + L.v1 * n[1], vnR = R.v0 * n[0] + R.v1 * n[1];
    const T HL = L.E + L.p * L.inv_rho, HR = R.E + R.p * R.inv_rho;
    const T sL = sqrt(L.rho), sR = sqrt(R.rho), inv = T(1.0) / (sL + sR);
    const T rt = sL * sR;
    const T ut0 = (sL * L.v0 + sR * R.v0) * inv, ut1 = (sL * L.v1 + sR * R.v1) * inv;
    const T Ht = (sL * HL + sR * HR) * inv;
    const T qq = ut0 * ut0 + ut1 * ut1;
    const T c2 = fmax((gam - T(1)) * (Ht - T(0.5) * qq), T(1e-14));
    const T ct = sqrt(c2);
    const T unt = ut0 * n[0] + ut1 * n[1];
    const T drho = R.rho - L.rho, dp = R.p - L.p, dun = vnR - vnL;
    const T dv0 = R.v0 - L.v0, dv1 = R.v1 - L.v1;
    const T delta = T(0.1) * ct;
    T l1 = fabs(unt - ct), l2 = fabs(unt), l4 = fabs(unt + ct);
    if (l1 < delta) l1 = (l1 * l1 + delta * delta) / (T(2) * delta);
    if (l4 < delta) l4 = (l4 * l4 + delta * delta) / (T(2) * delta);
    const T a1 = (dp - rt * ct * dun) / (T(2) * c2);
    const T a2 = drho - dp / c2;
    const T a4 = (dp + rt * ct * dun) / (T(2) * c2);
    const T s1 = l1 * a1, s2 = l2 * a2, s4 = l4 * a4, ss = l2 * rt;
    const T st0 = dv0 - dun * n[0], st1 = dv1 - dun * n[1];  // tangential velocity jump
    T d[4];
    d[0] = s1 + s2 + s4;
    d[1] = s1 * (ut0 - ct * n[0]) + s2 * ut0 + s4 * (ut0 + ct * n[0]) + ss * st0;
    d[2] = s1 * (ut1 - ct * n[1]) + s2 * ut1 + s4 * (ut1 + ct * n[1]) + ss * st1;
    d[3] = s1 * (Ht - ct * unt) + s2 * T(0.5) * qq + s4 * (Ht + ct * unt) + ss * (ut0 * st0 + ut1 * st1);
    const T fL[4] = {L.rho * vnL, L.mom0 * vnL + L.p * n[0], L.mom1 * vnL + L.p * n[1], vnL * (L.rhoE + L.p)};
    const T fR[4] = {R.rho * vnR, R.mom0 * vnR + R.p * n[0], R.mom1 * vnR + R.p * n[1], vnR * (R.rhoE + R.p)};
#pragma unroll
    for (int k = 0; k < 4; ++k) f[k] = T(0.5) * (fL[k] + fR[k]) - T(0.5) * d[k];
  }

  // the convective numerical flux the discretization selects
  template <class T>
  __device__ static inline void conv_sel(const PhysParams& pp, const T* uL, const T* uR, const T* n, T* f) {
    if (pp.ns_flux == ICX_FLUX_ROE) roe(pp, uL, uR, n, f);
    else conv(pp, uL, uR, n, f);
  }

  // exterior state of the PDE-level boundary kinds (apply_bc,
  // navier_stokes.hpp:976-1189). Slip wall: density and energy of the
  // interior, momentum mirrored about the wall. No-slip isothermal wall: the
  // interior density at rest with the wall temperature bval[0]. WALL_GENERAL:
  // the no-slip isothermal wall for a viscous discretization, else the slip
  // wall. Riemann (characteristic, Carlson NASA/TM-2011-217181): Riemann
  // invariants of the interior and the free stream, restated with the
  // reference's branches (its supersonic-outflow branch assigns a shadowing
  // local and so changes nothing; inflow takes R+ from the free stream),
  // then the boundary state from (rho, v, p).
  template <class T>
  __device__ static inline void apply_bc(const PhysParams& pp, const T* uL, const T* n, int bct, const double* bval,
                                         T* uR) {
    const T gam = T(pp.gamma);
    const T cp = gam / (gam - T(1)) * T(pp.Rgas);  // T_coeff with unit reference parameters
    NSState<T> L = ns_state(pp, uL);
    if (bct == ICX_BC_WALL_GENERAL) bct = pp.ns_viscous_wall ? ICX_BC_NO_SLIP_ISOTHERMAL : ICX_BC_SLIP_WALL;
    if (bct == ICX_BC_SLIP_WALL) {
      const T mn = L.mom0 * n[0] + L.mom1 * n[1];
      uR[0] = uL[0];
      uR[1] = L.mom0 - T(2) * mn * n[0];
      uR[2] = L.mom1 - T(2) * mn * n[1];
      uR[3] = uL[3];
    } else if (bct == ICX_BC_NO_SLIP_ISOTHERMAL) {
      const T rho = fmax(T(1e-14), L.rho);
      const T p = fmax(T(1e-12), rho * (gam - T(1)) / gam * cp * T(bval[0]));
      uR[0] = rho;
      uR[1] = T(0.0);
      uR[2] = T(0.0);
      uR[3] = rho * (p / (gam - T(1)) / rho);
    } else {  // ICX_BC_RIEMANN
      const T rho_o = fmax(T(1e-14), T(pp.fs_rho));
      const T p_o = fmax(T(1e-12), rho_o * (gam - T(1)) / gam * cp * T(pp.fs_T));
      const T c_o = sqrt(gam * p_o / rho_o);
      const T vn_i = L.v0 * n[0] + L.v1 * n[1];
      const T vn_o = T(pp.fs_u[0]) * n[0] + T(pp.fs_u[1]) * n[1];
      const T mach_n = vn_i / L.c;
      T rplus = vn_i + T(2) * L.c / (gam - T(1));
      const T rminus = vn_o - T(2) * c_o / (gam - T(1));
      if (mach_n < T(0)) rplus = vn_o + T(2) * c_o / (gam - T(1));
      const T ub = T(0.5) * (rplus + rminus);
      const T cb = T(0.25) * (gam - T(1)) * (rplus - rminus);
      const T vb0 = L.v0 + (ub - vn_i) * n[0], vb1 = L.v1 + (ub - vn_i) * n[1];
      const T sb = L.c * L.c / (gam * pow(L.rho, gam - T(1)));
      const T rhob = pow(cb * cb / (gam * sb), T(1.0) / (gam - T(1)));
      const T pb = rhob * cb * cb / gam;
      const T rho = fmax(T(1e-14), rhob), p = fmax(T(1e-12), pb);
      uR[0] = rho;
      uR[1] = vb0 * rho;
      uR[2] = vb1 * rho;
      uR[3] = rho * (p / (gam - T(1)) / rho + T(0.5) * (vb0 * vb0 + vb1 * vb1));
    }
  }
  static constexpr bool has_pde_bcs = true;

  // viscous normal flux; the energy term is mu*gamma/Pr * dE/dx_j n_j
  template <class T>
  __device__ static inline void diff(const PhysParams& pp, const T* u, const T* g, const T* n, T* f) {
    NSState<T> s = ns_state(pp, u);
    T tau[2][2], gv[2][2], gE[2], mgp;
    viscous(pp, s, g, tau, gv, gE, mgp);
    T vel[2] = {s.v0, s.v1};
    f[0] = f[1] = f[2] = f[3] = T(0.0);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      T ef = mgp * gE[j] * n[j];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        f[1 + i] += tau[i][j] * n[j];
        ef += vel[i] * tau[i][j] * n[j];
      }
      f[3] += ef;
    }
  }
  template <class T>
  __device__ static inline void neumann(const PhysParams&, const T*, T* f) {
    f[0] = f[1] = f[2] = f[3] = T(0.0);
  }
  static constexpr bool has_ic = false;  // no homogeneity tensor: no interface correction
};

}  // namespace icx
