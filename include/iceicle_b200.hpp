// C++23 host facade of iceicle_b200 over its C ABI (iceicle_b200.h), shaped
// like the reference's own templates so that a caller of the reference's
// residual / Jacobian / Newton path switches with few edits:
//
//   reference (iceicle)                                  here (iceicle_b200)
//   concepts physical_flux, convective_numerical_flux,   same names and call shapes
//     diffusion_flux, implements_bcs                       (conservation_law.hpp:20-90)
//   BurgersFlux / BurgersUpwind / BurgersDiffusionFlux   same names (burgers.hpp:41-250)
//   navier_stokes::Flux / VanLeer / DiffusionFlux        same names (navier_stokes.hpp:776-1301),
//                                                         plus navier_stokes::Roe
//   AbstractMesh{xmin, xmax, nelem, order, bct, bcflags} UniformMesh (same arguments)
//   FESpace{&mesh, LAGRANGE | LEGENDRE, GAUSS_LEGENDRE, p} FESpace{mesh, basis, p}
//   ConservationLawDDG{pflux, cflux, dflux} with public  ConservationLawDDG{pflux, cflux, dflux} with the
//     interior_penalty, sigma_ic, dirichlet_callbacks,     same public members (conservation_law.hpp:92-218)
//     neumann_callbacks, user_source
//   form_residual(fespace, disc, u, res)                 form_residual(fespace, disc, d_u, d_res)
//   form_petsc_jacobian_fd(fespace, disc, u, res, jac)   form_jacobian_fd(fespace, disc, d_u, d_res, jac)
//   ConvergenceCriteria, wolfe_linesearch,               same names and members
//     corrigan_linesearch, no_linesearch                   (nonlinear_solver_utils.hpp:24-268)
//   PetscNewton{fespace, disc, conv, ls}.solve(u)        NewtonSolver{fespace, disc, conv, ls}.solve(d_u)
//   CorriganLM{fespace, disc, conv, ls, geo_map}.solve(u) LMSolver{fespace, disc, conv, ls, geo_map}.solve(d_u)
//
// State and residual vectors are device pointers in the reference's
// fe_layout_right order ((element, basis function, equation)). The flux
// objects are evaluable on the host (they satisfy the concepts, so host code
// written against the reference's fluxes keeps working); the residual kernels
// evaluate the same formulas on the GPU, selected by the flux types. A flux
// type without a device implementation is rejected at compile time.
#pragma once

#include <array>
#include <cmath>
#include <concepts>
#include <functional>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

#include "iceicle_b200.h"

namespace iceicle_b200 {

// ------------------------------------------------------------------ errors
struct error : std::runtime_error {
  icx_status status;
  error(icx_status st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

inline void check(icx_status st, const icx_ctx* ctx, const char* what) {
  if (st == ICX_OK) return;
  std::string msg = std::string(what) + " failed (status " + std::to_string(st) + ")";
  if (ctx) {
    const char* e = icx_last_error(ctx);
    if (e && *e) msg += ": " + std::string(e);
  }
  throw error(st, msg);
}

// ------------------------------------------------------- small tensor types
// Tensor<T, n> and Tensor<T, n, m> as nested arrays (the reference uses
// NUMTOOL fixed-size tensors of the same shape)
template <class T, std::size_t N, std::size_t... M>
struct tensor_impl {
  using type = std::array<typename tensor_impl<T, M...>::type, N>;
};
template <class T, std::size_t N>
struct tensor_impl<T, N> {
  using type = std::array<T, N>;
};
template <class T, std::size_t... N>
using Tensor = typename tensor_impl<T, N...>::type;

// a read-only (neq x ndim) gradient, row-major: the role of the reference's
// mdspan<T, dextents<2>> gradient argument
template <class T>
struct grad_view {
  const T* data;
  int neq, ndim;
  constexpr T operator()(int eq, int d) const { return data[eq * ndim + d]; }
};

enum class BOUNDARY_CONDITIONS : int {
  PERIODIC = ICX_BC_PERIODIC,
  PARALLEL_COM = 1,
  NEUMANN = ICX_BC_NEUMANN,
  DIRICHLET = ICX_BC_DIRICHLET,
  EXTRAPOLATION = ICX_BC_EXTRAPOLATION,
  RIEMANN = ICX_BC_RIEMANN,
  NO_SLIP_ISOTHERMAL = ICX_BC_NO_SLIP_ISOTHERMAL,
  SLIP_WALL = ICX_BC_SLIP_WALL,
  WALL_GENERAL = ICX_BC_WALL_GENERAL,
  INLET = 9,
  OUTLET = 10,
  SPACETIME_PAST = ICX_BC_SPACETIME_PAST,
  SPACETIME_FUTURE = ICX_BC_SPACETIME_FUTURE,
  INTERIOR = ICX_BC_INTERIOR,
};

// ---------------------------------------------------------------- concepts
// the reference's flux concepts (conservation_law.hpp:20-90), with the
// gradient passed as grad_view
template <class FluxT>
concept physical_flux = requires(FluxT flux, std::array<typename FluxT::value_type, FluxT::nv_comp> u,
                                 grad_view<typename FluxT::value_type> gradu) {
  { flux(u, gradu) } -> std::same_as<Tensor<typename FluxT::value_type, FluxT::nv_comp, FluxT::ndim>>;
};

template <class FluxT>
concept convective_numerical_flux =
    requires(FluxT flux, std::array<typename FluxT::value_type, FluxT::nv_comp> uL,
             std::array<typename FluxT::value_type, FluxT::nv_comp> uR,
             Tensor<typename FluxT::value_type, FluxT::ndim> unit_normal) {
      { flux(uL, uR, unit_normal) } -> std::same_as<std::array<typename FluxT::value_type, FluxT::nv_comp>>;
    };

template <class FluxT>
concept diffusion_flux = requires(FluxT flux, std::array<typename FluxT::value_type, FluxT::nv_comp> u,
                                  grad_view<typename FluxT::value_type> gradu,
                                  Tensor<typename FluxT::value_type, FluxT::ndim> unit_normal) {
  { flux(u, gradu, unit_normal) } -> std::same_as<std::array<typename FluxT::value_type, FluxT::nv_comp>>;
};

template <class FluxT>
concept implements_bcs = requires(FluxT flux, std::array<typename FluxT::value_type, FluxT::nv_comp>& uL,
                                  grad_view<typename FluxT::value_type> graduL,
                                  Tensor<typename FluxT::value_type, FluxT::ndim> unit_normal,
                                  BOUNDARY_CONDITIONS bctype, int bcflag) {
  { flux.apply_bc(uL, graduL, unit_normal, bctype, bcflag) } ->
      std::same_as<std::array<typename FluxT::value_type, FluxT::nv_comp>>;
};

// ------------------------------------------------------------ Burgers fluxes
// BurgersCoefficients / BurgersFlux / BurgersUpwind / BurgersDiffusionFlux
// (burgers.hpp:17-250): lambda = a + b u / 2, F = lambda u - mu grad u
struct BurgersCoefficients {
  double mu = 0.001;
  std::array<double, 2> a{0.0, 0.0};
  std::array<double, 2> b{0.0, 0.0};
};

struct BurgersFlux {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 1, neq = 1;
  BurgersCoefficients coeffs;
  Tensor<double, 1, 2> operator()(std::array<double, 1> u, grad_view<double> g) const {
    Tensor<double, 1, 2> F{};
    for (int d = 0; d < 2; ++d) F[0][d] = (coeffs.a[d] + 0.5 * coeffs.b[d] * u[0]) * u[0] - coeffs.mu * g(0, d);
    return F;
  }
};

struct BurgersUpwind {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 1, neq = 1;
  BurgersCoefficients coeffs;
  std::array<double, 1> operator()(std::array<double, 1> uL, std::array<double, 1> uR,
                                   Tensor<double, 2> n) const {
    // upwind side chosen by the averaged wave speed P = n . (a + b uavg / 2),
    // flux n . (a + b u / 2) u of that side's state
    const double uavg = 0.5 * (uL[0] + uR[0]);
    double P = 0.0;
    for (int d = 0; d < 2; ++d) P += n[d] * (coeffs.a[d] + 0.5 * coeffs.b[d] * uavg);
    const double uup = P > 0 ? uL[0] : uR[0];
    double fa = 0.0;
    for (int d = 0; d < 2; ++d) fa += n[d] * (coeffs.a[d] + 0.5 * coeffs.b[d] * uup);
    return {fa * uup};
  }
};

struct BurgersDiffusionFlux {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 1, neq = 1;
  BurgersCoefficients coeffs;
  std::array<double, 1> operator()(std::array<double, 1>, grad_view<double> g, Tensor<double, 2> n) const {
    return {coeffs.mu * (g(0, 0) * n[0] + g(0, 1) * n[1])};
  }
  std::array<double, 1> neumann_flux(std::array<double, 1> gradn) const { return {coeffs.mu * gradn[0]}; }
};

// ----------------------------------------------------- Navier-Stokes fluxes
namespace navier_stokes {

// DimensionlessSutherlands (navier_stokes.hpp:260-287): the ratios of
// Sutherland's constants to the reference viscosity and temperature
struct DimensionlessSutherlands {
  double mu_0 = 1.716e-5, T_0 = 273.1, T_s = 110.5;
  double mu_ratio = 1.716e-5, T_0_ratio = 273.1, T_s_ratio = 110.5;  // unit reference parameters
  DimensionlessSutherlands() = default;
  DimensionlessSutherlands(double ref_mu, double ref_T)
      : mu_ratio(mu_0 / ref_mu), T_0_ratio(T_0 / ref_T), T_s_ratio(T_s / ref_T) {}
  double operator()(double That) const {
    return mu_ratio * std::pow(That / T_0_ratio, 1.5) * (T_0_ratio + T_s_ratio) / (That + T_s_ratio);
  }
};

// the physics of navier_stokes::Physics with unit ReferenceParameters, an
// ideal gas (CaloricallyPerfectEoS) and a constant viscosity mu, or
// Sutherland's law when `sutherland` is set
struct Physics {
  double gamma = 1.4;
  double Pr = 0.72;
  double mu = 0.01;
  double Rgas = 287.052874;
  std::optional<DimensionlessSutherlands> sutherland{};
  std::vector<double> isothermal_temperatures{};
  struct FreeStream {
    double rho_inf = 1.0, u_inf = 0.0;
    std::array<double, 2> u_direction{1.0, 0.0};
    double temp_inf = 1.0;
  } free_stream{};

  struct State {
    double rho, v[2], vv, rhoE, E, p, c, T;
  };
  double viscosity(const State& s) const { return sutherland ? (*sutherland)(s.T) : mu; }
  bool viscous() const { return sutherland.has_value() || mu != 0.0; }
  State thermo(const std::array<double, 4>& u) const {
    State s{};
    s.rho = std::max(1e-14, u[0]);
    s.v[0] = u[1] / s.rho;
    s.v[1] = u[2] / s.rho;
    s.vv = s.v[0] * s.v[0] + s.v[1] * s.v[1];
    s.rhoE = u[3];
    s.E = s.rhoE / s.rho;
    s.p = std::max(1e-12, (gamma - 1) * s.rho * (s.E - 0.5 * s.vv));
    s.c = std::sqrt(gamma * s.p / s.rho);
    s.T = s.p / s.rho * gamma / (gamma - 1) / (gamma / (gamma - 1) * Rgas);
    return s;
  }
};

struct Flux {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 4, neq = 4;
  Physics physics;
  Tensor<double, 4, 2> operator()(std::array<double, 4> u, grad_view<double> g) const {
    const auto s = physics.thermo(u);
    Tensor<double, 4, 2> F{};
    double gv[2][2], gE[2], tau[2][2];
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) gv[i][j] = (g(1 + i, j) - s.v[i] * g(0, j)) / s.rho;
    for (int j = 0; j < 2; ++j) gE[j] = (g(3, j) - s.E * g(0, j)) / s.rho;
    const double div = gv[0][0] + gv[1][1];
    const double mu = physics.viscosity(s);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) tau[i][j] = mu * (gv[i][j] + gv[j][i]) - (i == j ? 2.0 / 3.0 * mu * div : 0.0);
    for (int j = 0; j < 2; ++j) {
      F[0][j] = u[1 + j];
      for (int i = 0; i < 2; ++i) F[1 + i][j] = u[1 + i] * s.v[j] + (i == j ? s.p : 0.0) - tau[i][j];
      double q = mu * physics.gamma / physics.Pr * (gE[j] - s.v[0] * gv[0][j] - s.v[1] * gv[1][j]);
      F[3][j] = s.v[j] * (s.rhoE + s.p) - (q + s.v[0] * tau[0][j] + s.v[1] * tau[1][j]);
    }
    return F;
  }
  // exterior state of the PDE-level boundaries (the device kernels form the
  // same state; see icx_physics.cuh)
  std::array<double, 4> apply_bc(std::array<double, 4>& uL, grad_view<double>, Tensor<double, 2> n,
                                 BOUNDARY_CONDITIONS bct, int bcflag) const {
    const auto s = physics.thermo(uL);
    const double gam = physics.gamma, cp = gam / (gam - 1) * physics.Rgas;
    if (bct == BOUNDARY_CONDITIONS::WALL_GENERAL)
      bct = physics.viscous() ? BOUNDARY_CONDITIONS::NO_SLIP_ISOTHERMAL : BOUNDARY_CONDITIONS::SLIP_WALL;
    if (bct == BOUNDARY_CONDITIONS::SLIP_WALL) {
      const double mn = uL[1] * n[0] + uL[2] * n[1];
      return {uL[0], uL[1] - 2 * mn * n[0], uL[2] - 2 * mn * n[1], uL[3]};
    }
    if (bct == BOUNDARY_CONDITIONS::NO_SLIP_ISOTHERMAL) {
      const double p = std::max(1e-12, s.rho * (gam - 1) / gam * cp * physics.isothermal_temperatures.at(bcflag));
      return {s.rho, 0.0, 0.0, s.rho * (p / (gam - 1) / s.rho)};
    }
    if (bct != BOUNDARY_CONDITIONS::RIEMANN) return uL;
    const auto& fs = physics.free_stream;
    const double rho_o = std::max(1e-14, fs.rho_inf);
    const double p_o = std::max(1e-12, rho_o * (gam - 1) / gam * cp * fs.temp_inf);
    const double c_o = std::sqrt(gam * p_o / rho_o);
    const double vn_i = s.v[0] * n[0] + s.v[1] * n[1];
    const double vn_o = fs.u_inf * (fs.u_direction[0] * n[0] + fs.u_direction[1] * n[1]);
    double rp = vn_i + 2 * s.c / (gam - 1);
    const double rm = vn_o - 2 * c_o / (gam - 1);
    if (vn_i / s.c < 0) rp = vn_o + 2 * c_o / (gam - 1);
    const double ub = 0.5 * (rp + rm), cb = 0.25 * (gam - 1) * (rp - rm);
    const double vb0 = s.v[0] + (ub - vn_i) * n[0], vb1 = s.v[1] + (ub - vn_i) * n[1];
    const double sb = s.c * s.c / (gam * std::pow(s.rho, gam - 1));
    const double rho = std::max(1e-14, std::pow(cb * cb / (gam * sb), 1.0 / (gam - 1)));
    const double p = std::max(1e-12, rho * cb * cb / gam);
    return {rho, rho * vb0, rho * vb1, rho * (p / (gam - 1) / rho + 0.5 * (vb0 * vb0 + vb1 * vb1))};
  }
};

// Van Leer flux vector splitting on the normal Mach number (VanLeer, navier_stokes.hpp:776-864)
struct VanLeer {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 4, neq = 4;
  Physics physics;
  std::array<double, 4> operator()(std::array<double, 4> uL, std::array<double, 4> uR, Tensor<double, 2> n) const {
    const auto L = physics.thermo(uL), R = physics.thermo(uR);
    const double g = physics.gamma;
    std::array<double, 4> f{};
    auto part = [&](const Physics::State& S, const std::array<double, 4>& u, double sign) {
      const double vn = S.v[0] * n[0] + S.v[1] * n[1], m = vn / S.c;
      const double fm = sign * S.rho * S.c * (m + sign) * (m + sign) / 4.0;
      f[0] += fm;
      for (int d = 0; d < 2; ++d) f[1 + d] += fm * (S.v[d] + n[d] * (-vn + sign * 2 * S.c) / g);
      const double t = (g - 1) * vn + sign * 2 * S.c;
      f[3] += fm * ((S.vv - vn * vn) / 2 + t * t / (2 * (g * g - 1)));
      (void)u;
    };
    auto full = [&](const Physics::State& S, const std::array<double, 4>& u) {
      const double vn = S.v[0] * n[0] + S.v[1] * n[1];
      f[0] += S.rho * vn;
      for (int d = 0; d < 2; ++d) f[1 + d] += u[1 + d] * vn + S.p * n[d];
      f[3] += vn * (S.rhoE + S.p);
    };
    const double mL = (L.v[0] * n[0] + L.v[1] * n[1]) / L.c, mR = (R.v[0] * n[0] + R.v[1] * n[1]) / R.c;
    if (mL > 1) full(L, uL);
    else if (mL >= -1) part(L, uL, 1.0);
    if (mR < -1) full(R, uR);
    else if (mR <= 1) part(R, uR, -1.0);
    return f;
  }
};

// Roe's approximate Riemann solver with Harten's entropy fix (no reference counterpart)
struct Roe {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 4, neq = 4;
  Physics physics;
  std::array<double, 4> operator()(std::array<double, 4> uL, std::array<double, 4> uR, Tensor<double, 2> n) const {
    const auto L = physics.thermo(uL), R = physics.thermo(uR);
    const double g = physics.gamma;
    const double vnL = L.v[0] * n[0] + L.v[1] * n[1], vnR = R.v[0] * n[0] + R.v[1] * n[1];
    const double sL = std::sqrt(L.rho), sR = std::sqrt(R.rho), rt = sL * sR;
    double ut[2];
    for (int d = 0; d < 2; ++d) ut[d] = (sL * L.v[d] + sR * R.v[d]) / (sL + sR);
    const double Ht = (sL * (L.E + L.p / L.rho) + sR * (R.E + R.p / R.rho)) / (sL + sR);
    const double qq = ut[0] * ut[0] + ut[1] * ut[1];
    const double c2 = std::max((g - 1) * (Ht - 0.5 * qq), 1e-14), ct = std::sqrt(c2);
    const double un = ut[0] * n[0] + ut[1] * n[1];
    const double dp = R.p - L.p, dun = vnR - vnL;
    const double dl = 0.1 * ct;
    auto fix = [&](double l) { l = std::fabs(l); return l < dl ? (l * l + dl * dl) / (2 * dl) : l; };
    const double l1 = fix(un - ct), l2 = std::fabs(un), l4 = fix(un + ct);
    const double a1 = (dp - rt * ct * dun) / (2 * c2), a2 = (R.rho - L.rho) - dp / c2, a4 = (dp + rt * ct * dun) / (2 * c2);
    const double st[2] = {(R.v[0] - L.v[0]) - dun * n[0], (R.v[1] - L.v[1]) - dun * n[1]};
    std::array<double, 4> d{};
    d[0] = l1 * a1 + l2 * a2 + l4 * a4;
    for (int k = 0; k < 2; ++k)
      d[1 + k] = l1 * a1 * (ut[k] - ct * n[k]) + l2 * a2 * ut[k] + l4 * a4 * (ut[k] + ct * n[k]) + l2 * rt * st[k];
    d[3] = l1 * a1 * (Ht - ct * un) + l2 * a2 * 0.5 * qq + l4 * a4 * (Ht + ct * un) + l2 * rt * (ut[0] * st[0] + ut[1] * st[1]);
    const std::array<double, 4> fL{L.rho * vnL, uL[1] * vnL + L.p * n[0], uL[2] * vnL + L.p * n[1], vnL * (L.rhoE + L.p)};
    const std::array<double, 4> fR{R.rho * vnR, uR[1] * vnR + R.p * n[0], uR[2] * vnR + R.p * n[1], vnR * (R.rhoE + R.p)};
    std::array<double, 4> f{};
    for (int k = 0; k < 4; ++k) f[k] = 0.5 * (fL[k] + fR[k]) - 0.5 * d[k];
    return f;
  }
};

// the viscous normal flux (DiffusionFlux, navier_stokes.hpp:1241-1289)
struct DiffusionFlux {
  using value_type = double;
  static constexpr int ndim = 2, nv_comp = 4, neq = 4;
  Physics physics;
  // tau . n for the momentum, (mu gamma / Pr grad E + v . tau) . n for the
  // energy: the reference's diffusive flux carries the gradient of the total
  // energy (not of the internal energy) in its heat-flux term
  std::array<double, 4> operator()(std::array<double, 4> u, grad_view<double> g, Tensor<double, 2> n) const {
    const auto s = physics.thermo(u);
    double gv[2][2], gE[2], tau[2][2];
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) gv[i][j] = (g(1 + i, j) - s.v[i] * g(0, j)) / s.rho;
    for (int j = 0; j < 2; ++j) gE[j] = (g(3, j) - s.E * g(0, j)) / s.rho;
    const double div = gv[0][0] + gv[1][1];
    const double mu = physics.viscosity(s);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) tau[i][j] = mu * (gv[i][j] + gv[j][i]) - (i == j ? 2.0 / 3.0 * mu * div : 0.0);
    std::array<double, 4> f{};
    for (int j = 0; j < 2; ++j) {
      f[1] += tau[0][j] * n[j];
      f[2] += tau[1][j] * n[j];
      f[3] += (mu * physics.gamma / physics.Pr * gE[j] + s.v[0] * tau[0][j] + s.v[1] * tau[1][j]) * n[j];
    }
    return f;
  }
  std::array<double, 4> neumann_flux(std::array<double, 4>) const { return {0.0, 0.0, 0.0, 0.0}; }
};

}  // namespace navier_stokes

// which device physics a flux triple selects (a user-defined flux triple
// without a device implementation has no specialisation and is rejected)
template <class PF, class CF, class DF>
struct device_physics;
template <>
struct device_physics<BurgersFlux, BurgersUpwind, BurgersDiffusionFlux> {
  static void apply(icx_ctx* c, const BurgersFlux& pf, const BurgersUpwind&, const BurgersDiffusionFlux&) {
    check(icx_disc_burgers(c, pf.coeffs.mu, pf.coeffs.a.data(), pf.coeffs.b.data()), c, "icx_disc_burgers");
  }
};
template <class CF>
  requires(std::same_as<CF, navier_stokes::VanLeer> || std::same_as<CF, navier_stokes::Roe>)
struct device_physics<navier_stokes::Flux, CF, navier_stokes::DiffusionFlux> {
  static void apply(icx_ctx* c, const navier_stokes::Flux& pf, const CF&, const navier_stokes::DiffusionFlux&) {
    const auto& ph = pf.physics;
    const int kind = std::same_as<CF, navier_stokes::Roe> ? ICX_FLUX_ROE : ICX_FLUX_VANLEER;
    check(icx_disc_navier_stokes(c, ph.gamma, ph.Pr, ph.mu, kind), c, "icx_disc_navier_stokes");
    if (ph.sutherland)
      check(icx_disc_ns_viscosity(c, 1, ph.sutherland->mu_ratio, ph.sutherland->T_0_ratio, ph.sutherland->T_s_ratio),
            c, "icx_disc_ns_viscosity");
    check(icx_disc_ns_boundary(c, ph.isothermal_temperatures.data(), (int)ph.isothermal_temperatures.size(),
                               ph.free_stream.rho_inf, ph.free_stream.u_inf, ph.free_stream.u_direction.data(),
                               ph.free_stream.temp_inf, ph.Rgas),
          c, "icx_disc_ns_boundary");
  }
};

// ------------------------------------------------------- mesh and FE space
enum class FESPACE_BASIS { LAGRANGE = ICX_BASIS_LAGRANGE, LEGENDRE = ICX_BASIS_LEGENDRE };

// AbstractMesh{xmin, xmax, nelem, geometry order, bctypes, bcflags}: the
// uniform hypercube mesh of the reference's constructor (mesh.hpp:553-913);
// coord can be moved afterwards (perturbation, MDG node updates)
struct UniformMesh {
  std::array<double, 2> xmin, xmax;
  std::array<int, 2> nelem;
  int order;
  std::array<BOUNDARY_CONDITIONS, 4> bctypes;
  std::array<int, 4> bcflags;
  std::vector<std::array<double, 2>> coord;  // geometry nodes, x fastest

  UniformMesh(std::array<double, 2> xmin_, std::array<double, 2> xmax_, std::array<int, 2> nelem_, int order_,
              std::array<BOUNDARY_CONDITIONS, 4> bct, std::array<int, 4> bcf)
      : xmin(xmin_), xmax(xmax_), nelem(nelem_), order(order_), bctypes(bct), bcflags(bcf) {
    const int nnx = nelem[0] * order + 1, nny = nelem[1] * order + 1;
    coord.resize((std::size_t)nnx * nny);
    for (int j = 0; j < nny; ++j)
      for (int i = 0; i < nnx; ++i)
        coord[(std::size_t)j * nnx + i] = {xmin[0] + (xmax[0] - xmin[0]) * i / (nelem[0] * order),
                                           xmin[1] + (xmax[1] - xmin[1]) * j / (nelem[1] * order)};
  }
};

// FESpace{&mesh, basis, GAUSS_LEGENDRE, p}: owns the device context of the
// mesh and the space; the discretization is attached by the free functions
class FESpace {
 public:
  FESpace(UniformMesh& mesh, FESPACE_BASIS basis, int p, int device = 0) : mesh_(&mesh), basis_(basis), p_(p) {
    icx_ctx* c = nullptr;
    check(icx_create(&c, device), nullptr, "icx_create");
    ctx_.reset(c);
    int bct[4], bcf[4];
    for (int i = 0; i < 4; ++i) {
      bct[i] = (int)mesh.bctypes[i];
      bcf[i] = mesh.bcflags[i];
    }
    check(icx_mesh_uniform(c, 2, mesh.nelem.data(), mesh.xmin.data(), mesh.xmax.data(), mesh.order, bct, bcf), c,
          "icx_mesh_uniform");
    sync_coords();
    check(icx_fespace_basis(c, p, (int)basis), c, "icx_fespace_basis");
  }
  // after moving mesh.coord
  void sync_coords() {
    check(icx_mesh_set_coords(ctx_.get(), mesh_->coord.data()->data()), ctx_.get(), "icx_mesh_set_coords");
  }
  icx_ctx* ctx() const { return ctx_.get(); }
  const void* attached() const { return attached_; }
  void attach(const void* disc) { attached_ = disc; }
  icx_layout_info layout() const {
    icx_layout_info L{};
    check(icx_get_layout(ctx_.get(), &L), ctx_.get(), "icx_get_layout");
    return L;
  }
  int order() const { return p_; }

 private:
  struct Del {
    void operator()(icx_ctx* c) const { icx_destroy(c); }
  };
  UniformMesh* mesh_;
  FESPACE_BASIS basis_;
  int p_;
  std::unique_ptr<icx_ctx, Del> ctx_;
  const void* attached_ = nullptr;
};

// ------------------------------------------------------ the discretization
// ConservationLawDDG<PFlux, CFlux, DFlux> (conservation_law.hpp:92-218): the
// three fluxes and the reference's public members. Callbacks are evaluated
// on the host at the boundary and volume quadrature points when the space is
// set up (device kernels read the tables).
template <physical_flux PFlux, convective_numerical_flux CFlux, diffusion_flux DFlux>
class ConservationLawDDG {
 public:
  using value_type = typename PFlux::value_type;
  static constexpr int nv_comp = PFlux::nv_comp;
  static constexpr int dimensionality = PFlux::ndim;
  using callback = std::function<void(const value_type*, value_type*)>;

  PFlux phys_flux;
  CFlux conv_nflux;
  DFlux diff_flux;
  bool interior_penalty = false;
  value_type sigma_ic = 0.0;
  std::vector<callback> dirichlet_callbacks;
  std::vector<callback> neumann_callbacks;
  std::optional<callback> user_source;
  std::vector<std::string> field_names, residual_names;

  ConservationLawDDG(PFlux pf, CFlux cf, DFlux df)
      : phys_flux(std::move(pf)), conv_nflux(std::move(cf)), diff_flux(std::move(df)) {
    static_assert(requires { device_physics<PFlux, CFlux, DFlux>::apply; },
                  "this flux triple has no device implementation in iceicle_b200");
  }

  // pushes the discretization into the space's context and sets it up
  void setup(FESpace& fespace) {
    icx_ctx* c = fespace.ctx();
    device_physics<PFlux, CFlux, DFlux>::apply(c, phys_flux, conv_nflux, diff_flux);
    check(icx_disc_options(c, interior_penalty ? 1 : 0, sigma_ic), c, "icx_disc_options");
    for (std::size_t i = 0; i < dirichlet_callbacks.size(); ++i)
      check(icx_disc_dirichlet(c, (int)i, &trampoline, &dirichlet_callbacks[i]), c, "icx_disc_dirichlet");
    for (std::size_t i = 0; i < neumann_callbacks.size(); ++i)
      check(icx_disc_neumann(c, (int)i, &trampoline, &neumann_callbacks[i]), c, "icx_disc_neumann");
    if (user_source) check(icx_disc_source(c, &trampoline, &*user_source), c, "icx_disc_source");
    check(icx_setup(c), c, "icx_setup");
    fespace.attach(this);
  }

 private:
  static void trampoline(const double* x, double* out, void* f) { (*static_cast<callback*>(f))(x, out); }
};

template <class PF, class CF, class DF>
ConservationLawDDG(PF, CF, DF) -> ConservationLawDDG<PF, CF, DF>;

namespace detail {
template <class Disc>
icx_ctx* ready(FESpace& fespace, Disc& disc) {
  if (fespace.attached() != &disc) disc.setup(fespace);
  return fespace.ctx();
}
}  // namespace detail

// form_residual(fespace, disc, u, res) (form_residual.hpp:56-268)
template <class Disc>
void form_residual(FESpace& fespace, Disc& disc, const double* d_u, double* d_res, void* stream = nullptr) {
  icx_ctx* c = detail::ready(fespace, disc);
  check(icx_form_residual(c, d_u, d_res, stream), c, "icx_form_residual");
}

// the FD Jacobian in block-sparse rows (form_petsc_jacobian_fd,
// form_petsc_jacobian.hpp:55-317): host pattern, device values
struct BsrMatrix {
  int n_block_rows = 0, block_size = 0;
  std::vector<int> rowptr, colidx;
  double* d_vals = nullptr;  // nnz_blocks * bs * bs device doubles, owned by the caller
};

template <class Disc>
void jacobian_pattern(FESpace& fespace, Disc& disc, BsrMatrix& J) {
  icx_ctx* c = detail::ready(fespace, disc);
  const icx_layout_info L = fespace.layout();
  J.n_block_rows = L.n_elem;
  J.block_size = L.block_size;
  J.rowptr.resize(L.n_elem + 1);
  J.colidx.resize(L.nnz_blocks);
  check(icx_jacobian_pattern(c, J.rowptr.data(), J.colidx.data()), c, "icx_jacobian_pattern");
}

template <class Disc>
void form_jacobian_fd(FESpace& fespace, Disc& disc, const double* d_u, double* d_res, BsrMatrix& J, double eps = 0.0,
                      void* stream = nullptr) {
  icx_ctx* c = detail::ready(fespace, disc);
  check(icx_form_jacobian_fd(c, d_u, d_res, J.d_vals, eps, stream), c, "icx_form_jacobian_fd");
}

// the same Jacobian with the flux quadrature in FP32 (the reference's
// USE_SINGLE_PRECISION build of this call): FP32 values into d_vals32
// (nnz_blocks * bs * bs device floats), d_res = R(u) in FP64
template <class Disc>
void form_jacobian_fd_f32(FESpace& fespace, Disc& disc, const double* d_u, double* d_res, float* d_vals32,
                          void* stream = nullptr) {
  icx_ctx* c = detail::ready(fespace, disc);
  check(icx_form_jacobian_fd_f32(c, d_u, d_res, d_vals32, stream), c, "icx_form_jacobian_fd_f32");
}

// ------------------------------------------------------------------ solvers
// ConvergenceCriteria and the line searches (nonlinear_solver_utils.hpp:24-268)
struct ConvergenceCriteria {
  double tau_abs = 1e-8;
  double tau_rel = 1e-8;
  int kmax = 100;
  double r0 = 0.0;  // set by the solver
};
struct no_linesearch {};
struct wolfe_linesearch {
  int max_it = 20;
  double alpha_initial = 1, alpha_max = 10, c1 = 1e-4, c2 = 0.9;
};
struct corrigan_linesearch {
  int max_it = 20;
  double alpha_initial = 1, alpha_max = 10, alpha_min = 0;
};
using LinesearchVariant = std::variant<no_linesearch, corrigan_linesearch, wolfe_linesearch>;

// PetscNewton{fespace, disc, conv, ls}.solve(u) (petsc_newton.hpp:148-329):
// FD Jacobian, GMRES + block-ILU(0), the line search; the KSP settings are
// the members below (PETSc options in the reference)
template <class Disc>
class NewtonSolver {
 public:
  FESpace& fespace;
  Disc& disc;
  ConvergenceCriteria& conv_criteria;
  LinesearchVariant linesearch;
  icx_newton_options options{};
  icx_newton_report report{};

  NewtonSolver(FESpace& fs, Disc& d, ConvergenceCriteria& conv, LinesearchVariant ls = no_linesearch{})
      : fespace(fs), disc(d), conv_criteria(conv), linesearch(ls) {
    check(icx_newton_default_options(&options), nullptr, "icx_newton_default_options");
  }

  // u (device, fe_layout_right) updated in place; returns the iterations
  int solve(double* d_u) {
    icx_ctx* c = detail::ready(fespace, disc);
    options.tau_abs = conv_criteria.tau_abs;
    options.tau_rel = conv_criteria.tau_rel;
    options.kmax = conv_criteria.kmax;
    std::visit(
        [&](const auto& ls) {
          using L = std::decay_t<decltype(ls)>;
          if constexpr (std::same_as<L, no_linesearch>) {
            options.linesearch = 0;
          } else if constexpr (std::same_as<L, wolfe_linesearch>) {
            options.linesearch = 1;
            options.ls_max_it = ls.max_it;
            options.ls_alpha_initial = ls.alpha_initial;
            options.ls_alpha_max = ls.alpha_max;
            options.ls_c1 = ls.c1;
            options.ls_c2 = ls.c2;
          } else {
            options.linesearch = 2;
            options.ls_max_it = ls.max_it;
            options.ls_alpha_initial = ls.alpha_initial;
            options.ls_alpha_max = ls.alpha_max;
            options.ls_alpha_min = ls.alpha_min;
          }
        },
        linesearch);
    icx_status st = icx_newton_solve(c, d_u, &options, &report);
    if (st != ICX_ERR_NOT_CONVERGED) check(st, c, "icx_newton_solve");
    conv_criteria.r0 = report.r0;
    return report.iterations;
  }
};

// the geometry degrees of freedom of the selected traces (geo_dof_map,
// geo_layouts.hpp:359-540), with the hyper_rectangle boundary parametrisation
struct geo_dof_map {
  std::vector<int> traces;
  bool hyper_rectangle = true;
};

// CorriganLM{fespace, disc, conv, ls, geo_map}.solve(u) (corrigan_lm.hpp:112-717)
// with the reference's public regularisation members
template <class Disc>
class LMSolver {
 public:
  FESpace& fespace;
  Disc& disc;
  ConvergenceCriteria& conv_criteria;
  corrigan_linesearch linesearch;
  const geo_dof_map& geo_map;
  const bool explicitly_form_subproblem;
  double lambda_u = 1e-7, lambda_lag = 1e-5, lambda_b = 1e-2;
  icx_lm_options options{};
  icx_lm_report report{};
  std::vector<double> x;  // the geometry parameters (extract_geospan)

  LMSolver(FESpace& fs, Disc& d, ConvergenceCriteria& conv, corrigan_linesearch ls, const geo_dof_map& gm,
           bool explicitly_form_subproblem_ = false)
      : fespace(fs), disc(d), conv_criteria(conv), linesearch(ls), geo_map(gm),
        explicitly_form_subproblem(explicitly_form_subproblem_) {
    check(icx_lm_default_options(&options), nullptr, "icx_lm_default_options");
  }

  int solve(double* d_u) {
    icx_ctx* c = detail::ready(fespace, disc);
    check(icx_mdg_select(c, (int)geo_map.traces.size(), geo_map.traces.data(), geo_map.hyper_rectangle ? 1 : 0),
          c, "icx_mdg_select");
    int nsel = 0, ngeo = 0;
    check(icx_mdg_info(c, &nsel, &ngeo), c, "icx_mdg_info");
    x.resize(ngeo);
    check(icx_mdg_get_x(c, x.data()), c, "icx_mdg_get_x");
    options.tau_abs = conv_criteria.tau_abs;
    options.tau_rel = conv_criteria.tau_rel;
    options.kmax = conv_criteria.kmax;
    options.lambda_u = lambda_u;
    options.lambda_b = lambda_b;
    options.lambda_lag = lambda_lag;
    options.explicit_subproblem = explicitly_form_subproblem ? 1 : 0;
    options.linesearch = 2;
    options.ls_max_it = linesearch.max_it;
    options.ls_alpha_initial = linesearch.alpha_initial;
    options.ls_alpha_max = linesearch.alpha_max;
    options.ls_alpha_min = linesearch.alpha_min;
    icx_status st = icx_lm_solve(c, d_u, x.data(), &options, &report);
    if (st != ICX_ERR_NOT_CONVERGED) check(st, c, "icx_lm_solve");
    conv_criteria.r0 = report.r0;
    return report.iterations;
  }
};

}  // namespace iceicle_b200
