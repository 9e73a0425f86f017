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

// ------------------------------------------------------------------ Burgers
template <> struct Phys<ICX_PDE_BURGERS> {
  static constexpr int NEQ = 1;

  // F_d = (a_d + b_d u / 2) u - mu_d du/dx_d, mu_0 = mu, mu_1 = mu_t (mu, or 0
  // in spacetime form where the second coordinate is time: a_1 = 1, b_1 = 0
  // give F_t = u, burgers.hpp:261-340)
  __device__ static inline void flux(const PhysParams& pp, const double* u, const double* g, double* F) {
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      double lam = pp.a[d] + 0.5 * pp.b[d] * u[0];
      F[d] = lam * u[0] - (d == 0 ? pp.mu : pp.mu_t) * g[d];
    }
  }
  // upwinding on the averaged wavespeed P = n.(a + b uavg / 2)
  __device__ static inline void conv(const PhysParams& pp, const double* uL, const double* uR, const double* n,
                                     double* f) {
    double uavg = 0.5 * (uL[0] + uR[0]);
    double P = 0.0;
#pragma unroll
    for (int d = 0; d < 2; ++d) P += n[d] * (pp.a[d] + 0.5 * pp.b[d] * uavg);
    double uup = (P > 0) ? uL[0] : uR[0];
    double fa = 0.0;
#pragma unroll
    for (int d = 0; d < 2; ++d) fa += n[d] * (pp.a[d] + 0.5 * pp.b[d] * uup);
    f[0] = fa * uup;
  }
  __device__ static inline void diff(const PhysParams& pp, const double* u, const double* g, const double* n,
                                     double* f) {
    f[0] = pp.mu * g[0] * n[0] + pp.mu_t * g[1] * n[1];
  }
  __device__ static inline void neumann(const PhysParams& pp, const double* gn, double* f) { f[0] = pp.mu * gn[0]; }
  static constexpr bool has_ic = true;  // homogeneity tensor G = mu * I
  __device__ static inline void conv_sel(const PhysParams& pp, const double* uL, const double* uR, const double* n,
                                         double* f) {
    conv(pp, uL, uR, n, f);
  }
  // the Burgers fluxes implement no PDE-level boundaries: those faces contribute nothing
  static constexpr bool has_pde_bcs = false;
  __device__ static inline void apply_bc(const PhysParams&, const double* uL, const double*, int, const double*,
                                         double* uR) {
    uR[0] = uL[0];
  }
};

// ------------------------------------------------------------ Navier-Stokes
struct NSState {
  double rho, mom0, mom1, rhoE, v0, v1, vv, p, c, E, inv_rho;
};

constexpr double NS_RGAS = 287.052874;

// Quotients by the density are taken as products with one reciprocal per
// state (a last-bit difference from dividing each time).
__device__ static inline NSState ns_state(const PhysParams& pp, const double* u) {
  NSState s;
  double gamma = pp.gamma;
  s.rho = fmax(1e-14, u[0]);
  s.inv_rho = 1.0 / s.rho;
  s.mom0 = u[1];
  s.mom1 = u[2];
  s.v0 = u[1] * s.inv_rho;
  s.v1 = u[2] * s.inv_rho;
  s.vv = s.v0 * s.v0 + s.v1 * s.v1;
  s.rhoE = u[3];
  s.E = s.rhoE * s.inv_rho;
  double e = s.E - 0.5 * s.vv;
  s.p = fmax(1e-12, (gamma - 1) * s.rho * e);
  s.c = sqrt(gamma * s.p * s.inv_rho);
  return s;
}

template <> struct Phys<ICX_PDE_NAVIER_STOKES> {
  static constexpr int NEQ = 4;

  // velocity gradients gv[i][j] and total energy gradient gE[j]; shear stress
  __device__ static inline void viscous(const PhysParams& pp, const NSState& s, const double* g, double tau[2][2],
                                        double gv[2][2], double gE[2]) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) gv[i][j] = (g[2 * (1 + i) + j] - (i == 0 ? s.v0 : s.v1) * g[j]) * s.inv_rho;
#pragma unroll
    for (int j = 0; j < 2; ++j) gE[j] = (g[6 + j] - s.E * g[j]) * s.inv_rho;
    double mu = pp.ns_mu;
    double div = gv[0][0] + gv[1][1];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) tau[i][j] = mu * (gv[i][j] + gv[j][i]);
    tau[0][0] -= 2.0 / 3.0 * mu * div;
    tau[1][1] -= 2.0 / 3.0 * mu * div;
  }

  __device__ static inline void flux(const PhysParams& pp, const double* u, const double* g, double* F) {
    NSState s = ns_state(pp, u);
    double vel[2] = {s.v0, s.v1}, mom[2] = {s.mom0, s.mom1};
    // F[eq*2 + j]
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      F[0 * 2 + j] = mom[j];
#pragma unroll
      for (int i = 0; i < 2; ++i) F[(1 + i) * 2 + j] = mom[i] * vel[j];
      F[(1 + j) * 2 + j] += s.p;
      F[3 * 2 + j] = vel[j] * (s.rhoE + s.p);
    }
    double tau[2][2], gv[2][2], gE[2];
    viscous(pp, s, g, tau, gv, gE);
    double mu = pp.ns_mu;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double q = gE[j];
      q -= vel[0] * gv[0][j];
      q -= vel[1] * gv[1][j];
      q *= pp.mu_gamma_pr;
      double ef = q;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        F[(1 + i) * 2 + j] -= tau[i][j];
        ef += vel[i] * tau[i][j];
      }
      F[3 * 2 + j] -= ef;
    }
  }

  // Van Leer flux vector splitting on the normal Mach number
  __device__ static inline void conv(const PhysParams& pp, const double* uL, const double* uR, const double* n,
                                     double* f) {
    NSState L = ns_state(pp, uL), R = ns_state(pp, uR);
    double gam = pp.gamma;
    double vnL = L.v0 * n[0] + L.v1 * n[1];
    double vnR = R.v0 * n[0] + R.v1 * n[1];
    double mL = vnL / L.c, mR = vnR / R.c;
    const double inv_gam = pp.inv_gamma, inv_g21 = pp.inv_2gam2m1;
    if (mL > 1) {
      f[0] = L.rho * vnL;
      f[1] = L.mom0 * vnL + L.p * n[0];
      f[2] = L.mom1 * vnL + L.p * n[1];
      f[3] = vnL * (L.rhoE + L.p);
    } else if (mL < -1) {
      f[0] = f[1] = f[2] = f[3] = 0.0;
    } else {
      double fmL = L.rho * L.c * (mL + 1) * (mL + 1) / 4.0;
      f[0] = fmL;
      f[1] = fmL * (L.v0 + n[0] * (-vnL + 2 * L.c) * inv_gam);
      f[2] = fmL * (L.v1 + n[1] * (-vnL + 2 * L.c) * inv_gam);
      double t = (gam - 1) * vnL + 2 * L.c;
      f[3] = fmL * ((L.vv - vnL * vnL) / 2 + t * t * inv_g21);
    }
    if (mR < -1) {
      f[0] += R.rho * vnR;
      f[1] += R.mom0 * vnR + R.p * n[0];
      f[2] += R.mom1 * vnR + R.p * n[1];
      f[3] += vnR * (R.rhoE + R.p);
    } else if (mR <= 1) {
      double fmR = -R.rho * R.c * (mR - 1) * (mR - 1) / 4.0;
      f[0] += fmR;
      f[1] += fmR * (R.v0 + n[0] * (-vnR - 2 * R.c) * inv_gam);
      f[2] += fmR * (R.v1 + n[1] * (-vnR - 2 * R.c) * inv_gam);
      double t = (gam - 1) * vnR - 2 * R.c;
      f[3] += fmR * ((R.vv - vnR * vnR) / 2 + t * t * inv_g21);
    }
  }

  // Roe's approximate Riemann solver (P. L. Roe, J. Comput. Phys. 43, 1981):
  // F = (F(uL).n + F(uR).n) / 2 - sum_k |lambda_k| alpha_k r_k / 2 over the
  // acoustic, entropy and shear waves of the Roe-averaged state, with
  // Harten's entropy fix on the acoustic eigenvalues
  // (|l| < d: (l^2 + d^2) / (2 d), d = 0.1 c~). Unit reference parameters
  // (Eu = e_coeff = 1), so the ideal-gas relations take their usual form.
  __device__ static inline void roe(const PhysParams& pp, const double* uL, const double* uR, const double* n,
                                    double* f) {
    NSState L = ns_state(pp, uL), R = ns_state(pp, uR);
    const double gam = pp.gamma;
    const double vnL = L.v0 * n[0] + L.v1 * n[1], vnR = R.v0 * n[0] + R.v1 * n[1];
    const double HL = L.E + L.p * L.inv_rho, HR = R.E + R.p * R.inv_rho;
    const double sL = sqrt(L.rho), sR = sqrt(R.rho), inv = 1.0 / (sL + sR);
    const double rt = sL * sR;
    const double ut0 = (sL * L.v0 + sR * R.v0) * inv, ut1 = (sL * L.v1 + sR * R.v1) * inv;
    const double Ht = (sL * HL + sR * HR) * inv;
    const double qq = ut0 * ut0 + ut1 * ut1;
    const double c2 = fmax((gam - 1) * (Ht - 0.5 * qq), 1e-14);
    const double ct = sqrt(c2);
    const double unt = ut0 * n[0] + ut1 * n[1];
    const double drho = R.rho - L.rho, dp = R.p - L.p, dun = vnR - vnL;
    const double dv0 = R.v0 - L.v0, dv1 = R.v1 - L.v1;
    const double delta = 0.1 * ct;
    double l1 = fabs(unt - ct), l2 = fabs(unt), l4 = fabs(unt + ct);
    if (l1 < delta) l1 = (l1 * l1 + delta * delta) / (2 * delta);
    if (l4 < delta) l4 = (l4 * l4 + delta * delta) / (2 * delta);
    const double a1 = (dp - rt * ct * dun) / (2 * c2);
    const double a2 = drho - dp / c2;
    const double a4 = (dp + rt * ct * dun) / (2 * c2);
    const double s1 = l1 * a1, s2 = l2 * a2, s4 = l4 * a4, ss = l2 * rt;
    const double st0 = dv0 - dun * n[0], st1 = dv1 - dun * n[1];  // tangential velocity jump
    double d[4];
    d[0] = s1 + s2 + s4;
    d[1] = s1 * (ut0 - ct * n[0]) + s2 * ut0 + s4 * (ut0 + ct * n[0]) + ss * st0;
    d[2] = s1 * (ut1 - ct * n[1]) + s2 * ut1 + s4 * (ut1 + ct * n[1]) + ss * st1;
    d[3] = s1 * (Ht - ct * unt) + s2 * 0.5 * qq + s4 * (Ht + ct * unt) + ss * (ut0 * st0 + ut1 * st1);
    const double fL[4] = {L.rho * vnL, L.mom0 * vnL + L.p * n[0], L.mom1 * vnL + L.p * n[1], vnL * (L.rhoE + L.p)};
    const double fR[4] = {R.rho * vnR, R.mom0 * vnR + R.p * n[0], R.mom1 * vnR + R.p * n[1], vnR * (R.rhoE + R.p)};
#pragma unroll
    for (int k = 0; k < 4; ++k) f[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * d[k];
  }

  // the convective numerical flux the discretization selects
  __device__ static inline void conv_sel(const PhysParams& pp, const double* uL, const double* uR, const double* n,
                                         double* f) {
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
  __device__ static inline void apply_bc(const PhysParams& pp, const double* uL, const double* n, int bct,
                                         const double* bval, double* uR) {
    const double gam = pp.gamma;
    const double cp = gam / (gam - 1) * pp.Rgas;  // T_coeff with unit reference parameters
    NSState L = ns_state(pp, uL);
    if (bct == ICX_BC_WALL_GENERAL) bct = pp.ns_viscous_wall ? ICX_BC_NO_SLIP_ISOTHERMAL : ICX_BC_SLIP_WALL;
    if (bct == ICX_BC_SLIP_WALL) {
      const double mn = L.mom0 * n[0] + L.mom1 * n[1];
      uR[0] = uL[0];
      uR[1] = L.mom0 - 2 * mn * n[0];
      uR[2] = L.mom1 - 2 * mn * n[1];
      uR[3] = uL[3];
    } else if (bct == ICX_BC_NO_SLIP_ISOTHERMAL) {
      const double rho = fmax(1e-14, L.rho);
      const double p = fmax(1e-12, rho * (gam - 1) / gam * cp * bval[0]);
      uR[0] = rho;
      uR[1] = 0.0;
      uR[2] = 0.0;
      uR[3] = rho * (p / (gam - 1) / rho);
    } else {  // ICX_BC_RIEMANN
      const double rho_o = fmax(1e-14, pp.fs_rho);
      const double p_o = fmax(1e-12, rho_o * (gam - 1) / gam * cp * pp.fs_T);
      const double c_o = sqrt(gam * p_o / rho_o);
      const double vn_i = L.v0 * n[0] + L.v1 * n[1];
      const double vn_o = pp.fs_u[0] * n[0] + pp.fs_u[1] * n[1];
      const double mach_n = vn_i / L.c;
      double rplus = vn_i + 2 * L.c / (gam - 1);
      const double rminus = vn_o - 2 * c_o / (gam - 1);
      if (mach_n < 0) rplus = vn_o + 2 * c_o / (gam - 1);
      const double ub = 0.5 * (rplus + rminus);
      const double cb = 0.25 * (gam - 1) * (rplus - rminus);
      const double vb0 = L.v0 + (ub - vn_i) * n[0], vb1 = L.v1 + (ub - vn_i) * n[1];
      const double sb = L.c * L.c / (gam * pow(L.rho, gam - 1));
      const double rhob = pow(cb * cb / (gam * sb), 1.0 / (gam - 1));
      const double pb = rhob * cb * cb / gam;
      const double rho = fmax(1e-14, rhob), p = fmax(1e-12, pb);
      uR[0] = rho;
      uR[1] = vb0 * rho;
      uR[2] = vb1 * rho;
      uR[3] = rho * (p / (gam - 1) / rho + 0.5 * (vb0 * vb0 + vb1 * vb1));
    }
  }
  static constexpr bool has_pde_bcs = true;

  // viscous normal flux; the energy term is mu*gamma/Pr * dE/dx_j n_j
  __device__ static inline void diff(const PhysParams& pp, const double* u, const double* g, const double* n,
                                     double* f) {
    NSState s = ns_state(pp, u);
    double tau[2][2], gv[2][2], gE[2];
    viscous(pp, s, g, tau, gv, gE);
    double vel[2] = {s.v0, s.v1};
    f[0] = f[1] = f[2] = f[3] = 0.0;
    double mu = pp.ns_mu;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double ef = pp.mu_gamma_pr * gE[j] * n[j];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        f[1 + i] += tau[i][j] * n[j];
        ef += vel[i] * tau[i][j] * n[j];
      }
      f[3] += ef;
    }
  }
  __device__ static inline void neumann(const PhysParams&, const double*, double* f) {
    f[0] = f[1] = f[2] = f[3] = 0.0;
  }
  static constexpr bool has_ic = false;  // no homogeneity tensor: no interface correction
};

}  // namespace icx
