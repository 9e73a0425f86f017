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
