// Exercises the C++23 facade (include/iceicle_b200.hpp) the way a caller of
// the reference's templates would: mesh, space, ConservationLawDDG with the
// Burgers and Navier-Stokes flux objects, form_residual, the FD Jacobian and
// the Newton solver. Prints one line per result for the test to compare with
// the oracle:
//   residual <n> <v_0> ... <v_{n-1}>       Burgers 4 x 3 p = 2 residual at a given state
//   ns_residual <n> <v...>                 Navier-Stokes 3 x 3 p = 2, Roe flux, walls + far field
//   jacobian_blocks <nnzb> <bs>            BSR sizes of the Burgers Jacobian
//   jacobian_f32_rel <d>                   max |J_fp32 - J_fp64| / max |J_fp64| (FP32 flux quadrature)
//   newton <iterations> <|r_final|>        Burgers 8 x 8 Newton solve to 1e-10
// Usage: facade_check <state file: Burgers 4x3 p2 state (108 doubles)> <NS state file (144 doubles)>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <vector>

#include "iceicle_b200.hpp"

namespace ib = iceicle_b200;

static_assert(ib::physical_flux<ib::BurgersFlux>);
static_assert(ib::convective_numerical_flux<ib::BurgersUpwind>);
static_assert(ib::diffusion_flux<ib::BurgersDiffusionFlux>);
static_assert(ib::physical_flux<ib::navier_stokes::Flux>);
static_assert(ib::convective_numerical_flux<ib::navier_stokes::VanLeer>);
static_assert(ib::convective_numerical_flux<ib::navier_stokes::Roe>);
static_assert(ib::diffusion_flux<ib::navier_stokes::DiffusionFlux>);
static_assert(ib::implements_bcs<ib::navier_stokes::Flux>);
static_assert(!ib::implements_bcs<ib::BurgersFlux>);

static std::vector<double> read_doubles(const char* path, size_t n) {
  std::vector<double> v(n);
  std::ifstream f(path);
  for (auto& x : v) f >> x;
  return v;
}

static void print(const char* tag, const std::vector<double>& v) {
  std::printf("%s %zu", tag, v.size());
  for (double x : v) std::printf(" %.17g", x);
  std::printf("\n");
}

struct DeviceVec {
  double* p = nullptr;
  size_t n = 0;
  explicit DeviceVec(size_t n_) : n(n_) { cudaMalloc((void**)&p, n * sizeof(double)); }
  ~DeviceVec() { cudaFree(p); }
  void put(const std::vector<double>& h) { cudaMemcpy(p, h.data(), n * sizeof(double), cudaMemcpyHostToDevice); }
  std::vector<double> get() const {
    std::vector<double> h(n);
    cudaMemcpy(h.data(), p, n * sizeof(double), cudaMemcpyDeviceToHost);
    return h;
  }
};

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  using BC = ib::BOUNDARY_CONDITIONS;
  // Burgers 4 x 3, p = 2, geometry order 2, Dirichlet 0.25 on every side
  {
    ib::UniformMesh mesh({0.0, 0.0}, {1.0, 1.0}, {4, 3}, 2, {BC::DIRICHLET, BC::DIRICHLET, BC::DIRICHLET, BC::DIRICHLET},
                         {0, 0, 0, 0});
    ib::FESpace fespace(mesh, ib::FESPACE_BASIS::LAGRANGE, 2);
    ib::BurgersCoefficients coeffs{0.01, {0.3, -0.2}, {1.0, 0.5}};
    ib::ConservationLawDDG disc{ib::BurgersFlux{coeffs}, ib::BurgersUpwind{coeffs}, ib::BurgersDiffusionFlux{coeffs}};
    disc.dirichlet_callbacks.push_back([](const double*, double* out) { out[0] = 0.25; });
    const size_t n = 4 * 3 * 9;
    DeviceVec u(n), r(n);
    u.put(read_doubles(argv[1], n));
    ib::form_residual(fespace, disc, u.p, r.p);
    print("residual", r.get());
    ib::BsrMatrix J;
    ib::jacobian_pattern(fespace, disc, J);
    DeviceVec vals((size_t)J.rowptr.back() * J.block_size * J.block_size);
    J.d_vals = vals.p;
    ib::form_jacobian_fd(fespace, disc, u.p, r.p, J);
    std::printf("jacobian_blocks %d %d\n", J.rowptr.back(), J.block_size);
    // FP32 flux quadrature: largest block-entry difference to the FP64
    // Jacobian, relative to the largest entry
    float* v32 = nullptr;
    cudaMalloc((void**)&v32, vals.n * sizeof(float));
    ib::form_jacobian_fd_f32(fespace, disc, u.p, r.p, v32);
    std::vector<float> h32(vals.n);
    cudaMemcpy(h32.data(), v32, vals.n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(v32);
    const std::vector<double> h64 = vals.get();
    double dmax = 0.0, vmax = 0.0;
    for (size_t k = 0; k < h64.size(); ++k) {
      dmax = std::fmax(dmax, std::fabs((double)h32[k] - h64[k]));
      vmax = std::fmax(vmax, std::fabs(h64[k]));
    }
    std::printf("jacobian_f32_rel %.6e\n", dmax / vmax);
  }
  // Navier-Stokes 3 x 3, p = 2, Roe flux, Riemann far field left / right,
  // slip wall below, isothermal wall above (bcflag 1), Sutherland viscosity
  {
    ib::UniformMesh mesh({0.0, 0.0}, {1.0, 1.0}, {3, 3}, 2, {BC::RIEMANN, BC::SLIP_WALL, BC::RIEMANN, BC::NO_SLIP_ISOTHERMAL},
                         {0, 0, 0, 1});
    ib::FESpace fespace(mesh, ib::FESPACE_BASIS::LAGRANGE, 2);
    ib::navier_stokes::Physics ph;
    ph.isothermal_temperatures = {0.004, 0.005};
    ph.free_stream.rho_inf = 1.0;
    ph.free_stream.u_inf = 0.5;
    ph.free_stream.temp_inf = 0.004;
    ib::navier_stokes::DimensionlessSutherlands su;
    su.mu_ratio = 0.02;
    su.T_0_ratio = 0.004;
    su.T_s_ratio = 0.0015;
    ph.sutherland = su;
    ib::ConservationLawDDG disc{ib::navier_stokes::Flux{ph}, ib::navier_stokes::Roe{ph},
                                ib::navier_stokes::DiffusionFlux{ph}};
    disc.interior_penalty = true;
    const size_t n = 3 * 3 * 9 * 4;
    DeviceVec u(n), r(n);
    u.put(read_doubles(argv[2], n));
    ib::form_residual(fespace, disc, u.p, r.p);
    print("ns_residual", r.get());
  }
  // Burgers 8 x 8 Newton (Wolfe line search) from sin(2 pi x) sin(2 pi y) at the nodes
  {
    ib::UniformMesh mesh({0.0, 0.0}, {1.0, 1.0}, {8, 8}, 2, {BC::DIRICHLET, BC::DIRICHLET, BC::DIRICHLET, BC::DIRICHLET},
                         {0, 0, 0, 0});
    ib::FESpace fespace(mesh, ib::FESPACE_BASIS::LAGRANGE, 2);
    ib::BurgersCoefficients coeffs{0.01, {0.0, 0.0}, {1.0, 0.5}};
    ib::ConservationLawDDG disc{ib::BurgersFlux{coeffs}, ib::BurgersUpwind{coeffs}, ib::BurgersDiffusionFlux{coeffs}};
    disc.dirichlet_callbacks.push_back([](const double*, double* out) { out[0] = 0.0; });
    disc.setup(fespace);
    const size_t n = 8 * 8 * 9;
    std::vector<double> xy(2 * n);
    ib::check(icx_basis_node_coords(fespace.ctx(), xy.data()), fespace.ctx(), "icx_basis_node_coords");
    std::vector<double> u0(n);
    for (size_t k = 0; k < n; ++k) u0[k] = std::sin(2 * M_PI * xy[2 * k]) * std::sin(2 * M_PI * xy[2 * k + 1]);
    DeviceVec u(n);
    u.put(u0);
    ib::ConvergenceCriteria conv{1e-10, 0.0, 20};
    ib::NewtonSolver newton{fespace, disc, conv, ib::wolfe_linesearch{}};
    int k = newton.solve(u.p);
    std::printf("newton %d %.6e\n", k, newton.report.r_final);
    print("newton_state", u.get());
  }
  return 0;
}
