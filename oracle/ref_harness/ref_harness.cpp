// CPU reference build of the DG residual path: the reference project's own,
// unmodified headers (ConservationLawDDG, BurgersFlux/Upwind/DiffusionFlux,
// navier_stokes::Flux/VanLeer/DiffusionFlux, AbstractMesh, FESpace,
// form_residual, form_petsc_jacobian_fd) compiled against the project-written
// Numtool/PETSc stand-ins in this directory, exported through a small C ABI so
// that tests can call it with ctypes.
//
// Test infrastructure only: used to pin the oracle restatement and as the
// timed CPU baseline. Never linked into the product.
#include <chrono>
#include <functional>
#include <optional>
#include "iceicle/disc/conservation_law.hpp"
#include "iceicle/disc/burgers.hpp"
#include "iceicle/disc/navier_stokes.hpp"
#include "iceicle/fespace/fespace.hpp"
#include "iceicle/fe_function/fespan.hpp"
#include "iceicle/fe_function/layout_right.hpp"
#include "iceicle/form_residual.hpp"
#include "iceicle/fe_function/geo_layouts.hpp"
#include "iceicle/fe_function/component_span.hpp"
#ifdef REF_WITH_JACOBIAN
#include "iceicle/form_petsc_jacobian.hpp"
#endif
#include "iceicle/explicit_euler.hpp"
#include "iceicle/ssp_rk3.hpp"
#include "iceicle/tvd_rk3.hpp"
#include "iceicle/fe_function/restart.hpp"
#include "iceicle/pvd_writer.hpp"
#include <filesystem>
#include <cstring>
#include <functional>
#include <memory>
#include <vector>

using namespace iceicle;
using T = double;
using IDX = int;
static constexpr int ndim = 2;

extern "C" {
/// host callback for boundary data and sources: x[ndim] -> out[neq]
typedef void (*ref_point_fn)(const double* x, double* out, void* user);

/// problem description shared with the oracle restatement
struct ref_problem {
  int pde;              // 0: Burgers, 1: Navier-Stokes
  int nx, ny;
  int geo_order;
  int p;
  double xmin[2], xmax[2];
  int bctype[4];        // reference BOUNDARY_CONDITIONS values, order: left, bottom, right, top
  int bcflag[4];
  int interior_penalty;
  double sigma_ic;
  double mu;            // Burgers viscosity
  double a[2], b[2];    // Burgers linear / nonlinear advection
  double gamma, Pr;     // Navier-Stokes
  double ns_mu;         // constant viscosity
  int n_dirichlet;
  ref_point_fn dirichlet[8];
  void* dirichlet_user[8];
  int n_neumann;
  ref_point_fn neumann[8];
  void* neumann_user[8];
  ref_point_fn source;
  void* source_user;
  int spacetime;        // Burgers in (x, t): SpacetimeBurgersFlux / Upwind / Diffusion
  int basis;            // FESPACE_BASIS_TYPE of the solution space (0 LAGRANGE, 1 LEGENDRE)
  int ns_flux;          // 0 or 1: VanLeer (the reference has no other Navier-Stokes convective flux)
  int n_wall;           // Physics::isothermal_temperatures
  double wall_T[8];
  double fs_rho, fs_u_inf, fs_dir[2], fs_T;  // Physics::free_stream
  int ns_visc;                               // 0 constant_viscosity, 1 DimensionlessSutherlands
  double suth[3];                            // mu_ratio, T_0_ratio, T_s_ratio
};
}

namespace {

// Builds the uniform hypercube mesh with the reference's constructor and then
// writes the caller's node coordinates into it. The reference's uniform
// constructor sizes its 1D node lattice for geometry order 1 only
// (generate_directional_nodes makes nelem+1 points, the constructor reads
// nelem*order+1 of them); the lattice vectors are given enough capacity that
// those reads stay inside their allocations, and every coordinate is
// overwritten right after construction.
std::unique_ptr<AbstractMesh<T, IDX, ndim>> build_mesh(const ref_problem& pb, const double* coord) {
  std::array<std::vector<T>, ndim> nodes_1d;
  int nel[2] = {pb.nx, pb.ny};
  for (int d = 0; d < ndim; ++d) {
    int nfull = nel[d] * pb.geo_order + 1;
    std::vector<T> v;
    v.reserve(nfull);
    for (int i = 0; i < nfull; ++i)
      v.push_back(pb.xmin[d] + (pb.xmax[d] - pb.xmin[d]) * i / (nel[d] * pb.geo_order));
    v.resize(nel[d] + 1);  // capacity (and contents) of the full lattice kept
    nodes_1d[d] = std::move(v);
  }
  std::array<BOUNDARY_CONDITIONS, 4> bct;
  std::array<int, 4> bcf;
  for (int i = 0; i < 4; ++i) { bct[i] = (BOUNDARY_CONDITIONS)pb.bctype[i]; bcf[i] = pb.bcflag[i]; }
  auto mesh = std::make_unique<AbstractMesh<T, IDX, ndim>>(nodes_1d, pb.geo_order, bct, bcf);
  if (coord) {
    for (std::size_t i = 0; i < mesh->coord.size(); ++i) {
      mesh->coord[i][0] = coord[2 * i];
      mesh->coord[i][1] = coord[2 * i + 1];
    }
    mesh->update_coord_els();
  }
  return mesh;
}

template <class Disc>
void add_callbacks(Disc& disc, const ref_problem& pb) {
  for (int i = 0; i < pb.n_dirichlet; ++i) {
    ref_point_fn f = pb.dirichlet[i];
    void* u = pb.dirichlet_user[i];
    disc.dirichlet_callbacks.push_back([f, u](const T* x, T* out) { f(x, out, u); });
  }
  for (int i = 0; i < pb.n_neumann; ++i) {
    ref_point_fn f = pb.neumann[i];
    void* u = pb.neumann_user[i];
    disc.neumann_callbacks.push_back([f, u](const T* x, T* out) { f(x, out, u); });
  }
  if (pb.source) {
    ref_point_fn f = pb.source;
    void* u = pb.source_user;
    disc.user_source = std::function<void(const T*, T*)>{[f, u](const T* x, T* out) { f(x, out, u); }};
  }
  disc.interior_penalty = pb.interior_penalty != 0;
  disc.sigma_ic = pb.sigma_ic;
}

// runs `body(fespace, disc)` with the discretization of the problem
template <int P, class Body>
int with_disc(const ref_problem& pb, const double* coord, Body&& body) {
  auto mesh = build_mesh(pb, coord);
  FESpace<T, IDX, ndim> fespace{mesh.get(), pb.basis == 1 ? FESPACE_ENUMS::LEGENDRE : FESPACE_ENUMS::LAGRANGE,
                                FESPACE_ENUMS::GAUSS_LEGENDRE,
                                std::integral_constant<int, P>{}};
  if (pb.pde == 0 && pb.spacetime) {
    BurgersCoefficients<T, ndim - 1> coeffs{};
    coeffs.mu = pb.mu;
    coeffs.a[0] = pb.a[0];
    coeffs.b[0] = pb.b[0];
    SpacetimeBurgersFlux<T, ndim> pf{coeffs};
    SpacetimeBurgersUpwind<T, ndim> cf{coeffs};
    SpacetimeBurgersDiffusion<T, ndim> df{coeffs};
    ConservationLawDDG disc{std::move(pf), std::move(cf), std::move(df)};
    add_callbacks(disc, pb);
    return body(fespace, disc, std::integral_constant<std::size_t, 1>{});
  } else if (pb.pde == 0) {
    BurgersCoefficients<T, ndim> coeffs{};
    coeffs.mu = pb.mu;
    coeffs.a[0] = pb.a[0]; coeffs.a[1] = pb.a[1];
    coeffs.b[0] = pb.b[0]; coeffs.b[1] = pb.b[1];
    BurgersFlux pf{coeffs};
    BurgersUpwind cf{coeffs};
    BurgersDiffusionFlux df{coeffs};
    ConservationLawDDG disc{std::move(pf), std::move(cf), std::move(df)};
    add_callbacks(disc, pb);
    return body(fespace, disc, std::integral_constant<std::size_t, 1>{});
  } else {
    if (pb.ns_flux > 1) return -4;  // no Roe flux in the reference
    navier_stokes::ReferenceParameters<T> ref{};
    navier_stokes::CaloricallyPerfectEoS<T, ndim> eos{};
    eos.gamma = pb.gamma;
    navier_stokes::constant_viscosity<T> visc{pb.ns_mu};
    navier_stokes::DimensionlessSutherlands<T> suth{ref};
    suth.mu_ratio = pb.suth[0];
    suth.T_0_ratio = pb.suth[1];
    suth.T_s_ratio = pb.suth[2];
    auto make_physics = [&]() {
      if (pb.ns_visc == 1)
        return navier_stokes::Physics<T, ndim, navier_stokes::CaloricallyPerfectEoS<T, ndim>>{ref, eos, suth, pb.Pr};
      return navier_stokes::Physics<T, ndim, navier_stokes::CaloricallyPerfectEoS<T, ndim>>{ref, eos, visc, pb.Pr};
    };
    navier_stokes::Physics<T, ndim, navier_stokes::CaloricallyPerfectEoS<T, ndim>> physics = make_physics();
    // boundary data before the flux objects copy the physics
    physics.isothermal_temperatures.assign(pb.wall_T, pb.wall_T + pb.n_wall);
    physics.free_stream.rho_inf = pb.fs_rho;
    physics.free_stream.u_inf = pb.fs_u_inf;
    physics.free_stream.u_direction[0] = pb.fs_dir[0];
    physics.free_stream.u_direction[1] = pb.fs_dir[1];
    physics.free_stream.temp_inf = pb.fs_T;
    // the full Navier-Stokes flux for a viscous problem, the Euler one otherwise
    // (its WALL_GENERAL is the slip wall)
    auto run = [&](auto full_ns) {
      navier_stokes::Flux flux{physics, full_ns};
      navier_stokes::VanLeer numflux{physics};
      navier_stokes::DiffusionFlux dflux{physics, full_ns};
      ConservationLawDDG disc{std::move(flux), std::move(numflux), std::move(dflux)};
      add_callbacks(disc, pb);
      return body(fespace, disc, std::integral_constant<std::size_t, 4>{});
    };
    if (pb.ns_mu != 0.0 || pb.ns_visc == 1) return run(std::true_type{});
    return run(std::false_type{});
  }
}

// field and residual names the reference's applications give each PDE
// (conservation_law.cpp:246-247, ns_manufactured.cpp:246-257)
std::vector<std::string> field_names(int pde) {
  if (pde == 0) return {"u"};
  return {"rho", "rhou", "rhov", "rhoe"};
}
std::vector<std::string> residual_names(int pde) {
  if (pde == 0) return {"residual"};
  return {"density_conservation", "momentum_u_conservation", "momentum_v_conservation", "energy_conservation"};
}

// runs f with the working directory set to dir (the reference's writers
// write under std::filesystem::current_path())
template <class F>
int in_directory(const char* dir, F&& f) {
  auto old = std::filesystem::current_path();
  std::filesystem::current_path(dir);
  int rc = f();
  std::filesystem::current_path(old);
  return rc;
}

template <class Body>
int dispatch_p(const ref_problem& pb, const double* coord, Body&& body) {
  switch (pb.p) {
    case 1: return with_disc<1>(pb, coord, body);
    case 2: return with_disc<2>(pb, coord, body);
    case 3: return with_disc<3>(pb, coord, body);
    case 4: return with_disc<4>(pb, coord, body);
    default: return -1;
  }
}

}  // namespace

extern "C" {

/// number of mesh nodes of the uniform mesh of a problem
int ref_n_nodes(const ref_problem* pb) {
  return (pb->nx * pb->geo_order + 1) * (pb->ny * pb->geo_order + 1);
}

/// node coordinates of the unperturbed uniform mesh, x fastest
int ref_mesh_coords(const ref_problem* pb, double* coord_out) {
  auto mesh = build_mesh(*pb, nullptr);
  for (std::size_t i = 0; i < mesh->coord.size(); ++i) {
    coord_out[2 * i] = mesh->coord[i][0];
    coord_out[2 * i + 1] = mesh->coord[i][1];
  }
  return (int)mesh->coord.size();
}

/// Mesh topology as built by the reference: element node lists (conn_el,
/// nnode per element) and faces in reference order with
/// (elemL, elemR, face_nr_l, face_nr_r, orientation_r, bctype, bcflag).
/// Returns the number of faces; sizes: conn_out[nelem*nnode], face_out[nface*7].
int ref_mesh_topology(const ref_problem* pb, int* conn_out, int* face_out, int* n_interior_out) {
  auto mesh = build_mesh(*pb, nullptr);
  IDX nel = mesh->nelem();
  int k = 0;
  for (IDX e = 0; e < nel; ++e)
    for (std::size_t j = 0; j < mesh->conn_el.rowsize(e); ++j) conn_out[k++] = mesh->conn_el[e, j];
  int nf = (int)mesh->faces.size();
  for (int f = 0; f < nf; ++f) {
    const auto& fc = *mesh->faces[f];
    face_out[7 * f + 0] = fc.elemL;
    face_out[7 * f + 1] = fc.elemR;
    face_out[7 * f + 2] = (int)fc.face_nr_l();
    face_out[7 * f + 3] = (int)fc.face_nr_r();
    face_out[7 * f + 4] = (int)(fc.face_infoR % FACE_INFO_MOD);
    face_out[7 * f + 5] = (int)fc.bctype;
    face_out[7 * f + 6] = fc.bcflag;
  }
  *n_interior_out = (int)(mesh->interiorFaceEnd - mesh->interiorFaceStart);
  return nf;
}

/// form_residual(fespace, disc, u, res) of the reference
int ref_form_residual(const ref_problem* pb, const double* coord, const double* u, double* res) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::vector<T> ubuf(u, u + layout.size());
    std::vector<T> rbuf(layout.size());
    fespan uspan{ubuf.data(), layout};
    fespan rspan{rbuf.data(), layout};
    solvers::form_residual(fespace, disc, uspan, rspan);
    std::memcpy(res, rbuf.data(), sizeof(T) * rbuf.size());
    return 0;
  });
}

/// time `nrep` calls of form_residual (mesh, space and disc built once);
/// returns seconds per call through *seconds
int ref_time_form_residual(const ref_problem* pb, const double* coord, const double* u, int nrep,
                           double* seconds) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::vector<T> ubuf(u, u + layout.size());
    std::vector<T> rbuf(layout.size());
    fespan uspan{ubuf.data(), layout};
    fespan rspan{rbuf.data(), layout};
    solvers::form_residual(fespace, disc, uspan, rspan);  // warm-up
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < nrep; ++i) solvers::form_residual(fespace, disc, uspan, rspan);
    auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count() / nrep;
    return 0;
  });
}

/// MDG-ICE: geo_dof_map over the given traces (optionally with the
/// hyper_rectangle boundary parametrisation). Writes the selected node list,
/// the geometry parameters x (extract_geospan) and returns their count; the
/// caller sizes arrays with ref_n_nodes.
int ref_mdg_select(const ref_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                   int* n_selected, int* selected_nodes, double* x_out) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    std::vector<int> tr(traces, traces + ntr);
    geo_dof_map geo_map{tr, fespace};
    if (hyper)
      mesh_parameterizations::hyper_rectangle(std::array<int, 2>{pb->nx, pb->ny},
                                              std::array<double, 2>{pb->xmin[0], pb->xmin[1]},
                                              std::array<double, 2>{pb->xmax[0], pb->xmax[1]}, geo_map);
    *n_selected = (int)geo_map.selected_nodes.size();
    for (std::size_t i = 0; i < geo_map.selected_nodes.size(); ++i) selected_nodes[i] = geo_map.selected_nodes[i];
    geo_data_layout x_layout{geo_map};
    std::vector<T> xdata(x_layout.size());
    component_span x{xdata, x_layout};
    extract_geospan(*fespace.meshptr, x);
    std::memcpy(x_out, xdata.data(), sizeof(T) * xdata.size());
    return (int)xdata.size();
  });
}

/// form_residual(fespace, disc, geo_map, [u; x], [res; ic]) (form_residual.hpp:426-452)
int ref_mdg_residual(const ref_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                     const double* u_and_x, int n_total, double* res_and_ic, int n_res) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    std::vector<int> tr(traces, traces + ntr);
    geo_dof_map geo_map{tr, fespace};
    if (hyper)
      mesh_parameterizations::hyper_rectangle(std::array<int, 2>{pb->nx, pb->ny},
                                              std::array<double, 2>{pb->xmin[0], pb->xmin[1]},
                                              std::array<double, 2>{pb->xmax[0], pb->xmax[1]}, geo_map);
    std::vector<T> ux(u_and_x, u_and_x + n_total);
    std::vector<T> rr(n_res);
    solvers::form_residual(fespace, disc, geo_map, std::span<T>{ux}, std::span<T>{rr});
    std::memcpy(res_and_ic, rr.data(), sizeof(T) * n_res);
    return 0;
  });
}

#ifdef REF_WITH_JACOBIAN
/// MDG Jacobian of [res; ic] w.r.t. [u; x] (form_petsc_jacobian_fd followed by
/// form_petsc_mdg_jacobian_fd, the sparse path of CorriganLM::solve,
/// corrigan_lm.hpp:385-396) into a dense row-major (N + nic) x (N + ngeo) array
int ref_mdg_jacobian_dense(const ref_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                           const double* u, const double* x, int ngeo, double* res_and_ic, int nres,
                           double* jac_dense) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    std::vector<int> tr(traces, traces + ntr);
    geo_dof_map geo_map{tr, fespace};
    if (hyper)
      mesh_parameterizations::hyper_rectangle(std::array<int, 2>{pb->nx, pb->ny},
                                              std::array<double, 2>{pb->xmin[0], pb->xmin[1]},
                                              std::array<double, 2>{pb->xmax[0], pb->xmax[1]}, geo_map);
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::size_t n = layout.size();
    std::vector<T> ubuf(u, u + n);
    std::vector<T> rbuf(nres);
    fespan uspan{ubuf.data(), layout};
    fespan rspan{rbuf.data(), layout};
    geo_data_layout x_layout{geo_map};
    std::vector<T> xdata(x, x + ngeo);
    component_span xspan{xdata, x_layout};
    ic_residual_layout<T, IDX, ndim, decltype(neq_c)::value> ic_layout{geo_map};
    dofspan mdg_res{rbuf.data() + n, ic_layout};
    Mat jac;
    MatCreate(PETSC_COMM_WORLD, &jac);
    MatSetSizes(jac, (PetscInt)nres, (PetscInt)(n + ngeo), PETSC_DETERMINE, PETSC_DETERMINE);
    update_mesh(xspan, *fespace.meshptr);
    solvers::form_petsc_jacobian_fd(fespace, disc, uspan, rspan, jac);
    solvers::form_petsc_mdg_jacobian_fd(fespace, disc, uspan, xspan, mdg_res, jac);
    std::memcpy(res_and_ic, rbuf.data(), sizeof(T) * nres);
    petsc_shim_to_dense(jac, jac_dense);
    MatDestroy(&jac);
    return 0;
  });
}

/// time `nrep` calls of the reference's form_petsc_jacobian_fd (with its
/// residual) into preallocated block storage of the element pattern (rowptr
/// [E + 1], colidx: the element and its face neighbours, ascending); the
/// values of the last call are left in vals (nnzb blocks of bs x bs)
int ref_time_jacobian_fd(const ref_problem* pb, const double* coord, const double* u, const int* rowptr,
                         const int* colidx, double* vals, int nrep, double* seconds) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::size_t n = layout.size();
    const int E = pb->nx * pb->ny;
    const int bs = (int)(n / (std::size_t)E);
    std::vector<T> ubuf(u, u + n);
    std::vector<T> rbuf(n);
    fespan uspan{ubuf.data(), layout};
    fespan rspan{rbuf.data(), layout};
    Mat jac;
    MatCreate(PETSC_COMM_WORLD, &jac);
    MatSetSizes(jac, (PetscInt)n, (PetscInt)n, PETSC_DETERMINE, PETSC_DETERMINE);
    jac->bsr_vals = vals;
    jac->bsr_rowptr = rowptr;
    jac->bsr_colidx = colidx;
    jac->bs = bs;
    const std::size_t nv = (std::size_t)rowptr[E] * bs * bs;
    std::fill(vals, vals + nv, 0.0);
    solvers::form_petsc_jacobian_fd(fespace, disc, uspan, rspan, jac);  // warm-up
    auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < nrep; ++r) {
      std::fill(vals, vals + nv, 0.0);  // MatZeroEntries
      solvers::form_petsc_jacobian_fd(fespace, disc, uspan, rspan, jac);
    }
    auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count() / std::max(nrep, 1);
    MatDestroy(&jac);
    return 0;
  });
}

/// form_petsc_jacobian_fd of the reference into a dense row-major N x N
/// matrix (small meshes only), plus the residual
int ref_form_jacobian_dense(const ref_problem* pb, const double* coord, const double* u, double* res,
                            double* jac_dense) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::size_t n = layout.size();
    std::vector<T> ubuf(u, u + n);
    std::vector<T> rbuf(n);
    fespan uspan{ubuf.data(), layout};
    fespan rspan{rbuf.data(), layout};
    Mat jac;
    MatCreate(PETSC_COMM_WORLD, &jac);
    MatSetSizes(jac, (PetscInt)n, (PetscInt)n, PETSC_DETERMINE, PETSC_DETERMINE);
    solvers::form_petsc_jacobian_fd(fespace, disc, uspan, rspan, jac);
    std::memcpy(res, rbuf.data(), sizeof(T) * n);
    petsc_shim_to_dense(jac, jac_dense);
    MatDestroy(&jac);
    return 0;
  });
}
#endif


/// element mass matrices [E][nb][nb] (calculate_mass_matrix)
int ref_mass_matrices(const ref_problem* pb, const double* coord, double* M) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    size_t k = 0;
    for (const auto& el : fespace.elements) {
      auto mass = calculate_mass_matrix(el);
      const int nb = el.nbasis();
      for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) M[k++] = mass[i][j];
    }
    return 0;
  });
}

/// the reference's explicit solvers run to completion from u (updated in
/// place): scheme 0 ExplicitEuler, 1 RK3TVD, 2 RK3SSP; dt_kind 0 FixedTimestep,
/// 1 CFLTimestep (Burgers only); term_kind 0 TimestepTermination (ntime),
/// 1 TfinalTermination (tfinal)
int ref_explicit_solve(const ref_problem* pb, const double* coord, double* u, int scheme, int dt_kind, double dt,
                       double cfl, int term_kind, int ntime, double tfinal, int* steps_out, double* time_out) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) -> int {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::vector<T> ubuf(u, u + layout.size());
    fespan uspan{ubuf.data(), layout};
    auto with_stop = [&](auto timestep) -> int {
      auto with_scheme = [&](auto stop) -> int {
        auto go = [&](auto& solver) {
          solver.vis_callback = [](auto&) {};
          solver.solve(fespace, disc, uspan);
          *steps_out = solver.itime;
          *time_out = solver.time;
        };
        if (scheme == 0) { solvers::ExplicitEuler solver{fespace, disc, timestep, stop}; go(solver); }
        else if (scheme == 1) { solvers::RK3TVD solver{fespace, disc, timestep, stop}; go(solver); }
        else { solvers::RK3SSP solver{fespace, disc, timestep, stop}; go(solver); }
        return 0;
      };
      if (term_kind == 0) return with_scheme(solvers::TimestepTermination<T, IDX>{ntime});
      solvers::TfinalTermination<T, IDX> tf{};
      tf.tfinal = tfinal;
      return with_scheme(tf);
    };
    int rc = -2;
    if (dt_kind == 0) rc = with_stop(solvers::FixedTimestep<T, IDX>{dt});
    else if constexpr (requires { disc.dt_from_cfl(1.0, 1.0); }) {
      solvers::CFLTimestep<T, IDX> c{};
      c.cfl = cfl;
      rc = with_stop(c);
    }
    if (rc == 0) std::memcpy(u, ubuf.data(), sizeof(T) * ubuf.size());
    return rc;
  });
}

/// write_restart(fespace, u, k) (fe_function/restart.hpp:20-59) run in `dir`:
/// writes dir/RESTART/restart<k>_0
int ref_write_restart(const ref_problem* pb, const double* coord, const double* u, int k, const char* dir) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::vector<T> ubuf(u, u + layout.size());
    fespan uspan{ubuf.data(), layout};
    return in_directory(dir, [&] { write_restart(fespace, uspan, k); return 0; });
  });
}

/// read_restart(fespace, u, name) (restart.hpp:68-108) run in `dir`: the
/// node coordinates it leaves in the mesh and u
int ref_read_restart(const ref_problem* pb, const char* name, const char* dir, double* coord_out, double* u_out) {
  return dispatch_p(*pb, nullptr, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::vector<T> ubuf(layout.size());
    fespan uspan{ubuf.data(), layout};
    int rc = in_directory(dir, [&] { read_restart(fespace, uspan, std::string{name}); return 0; });
    const auto& c = fespace.meshptr->coord;
    for (std::size_t i = 0; i < c.size(); ++i) { coord_out[2 * i] = c[i][0]; coord_out[2 * i + 1] = c[i][1]; }
    std::memcpy(u_out, ubuf.data(), sizeof(T) * ubuf.size());
    return rc;
  });
}

/// PVDWriter::write_vtu(itime, itime) (io/pvd_writer.hpp:1095-1140) into
/// dir/<collection><itime>.vtu: kind 0 register_fields(u, field names),
/// kind 1 register_residuals(u, residual names, disc)
int ref_write_vtu(const ref_problem* pb, const double* coord, const double* u, int kind, int itime,
                  const char* dir, const char* collection) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    fe_layout_right layout{fespace.dg_map, neq_c};
    std::vector<T> ubuf(u, u + layout.size());
    fespan uspan{ubuf.data(), layout};
    io::PVDWriter<T, IDX, ndim> w{};
    w.data_directory = dir;
    w.collection_name = collection;
    w.register_fespace(fespace);
    if (kind == 0) w.register_fields(uspan, field_names(pb->pde));
    else w.register_residuals(uspan, residual_names(pb->pde), disc);
    w.write_vtu(itime, (T)itime);
    return 0;
  });
}

/// the MDG interface-conservation residual as the reference's implicit
/// driver writes it (solvers_lua_interface.hpp:589-632): ic ([selected node]
/// [neq], geo_dof_map order) scattered into an H1 field over the mesh nodes
/// and written by a PVDWriter on the geometry-order H1 space
int ref_write_vtu_mdg(const ref_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                      const double* ic, int itime, const char* dir, const char* collection) {
  return dispatch_p(*pb, coord, [&](auto& fespace, auto& disc, auto neq_c) {
    std::vector<int> tr(traces, traces + ntr);
    geo_dof_map geo_map{tr, fespace};
    if (hyper)
      mesh_parameterizations::hyper_rectangle(std::array<int, 2>{pb->nx, pb->ny},
                                              std::array<double, 2>{pb->xmin[0], pb->xmin[1]},
                                              std::array<double, 2>{pb->xmax[0], pb->xmax[1]}, geo_map);
    constexpr int NEQ = (int)decltype(neq_c)::value;
    FESpace space_h1{fespace.meshptr};
    fe_layout_right h1_layout{fespace.cg_map, tmp::to_size<NEQ>()};
    std::vector<T> h1_data(h1_layout.size());
    fespan res_mdg_h1{h1_data, h1_layout};
    ic_residual_layout<T, IDX, ndim, NEQ> ic_layout{geo_map};
    std::vector<T> icbuf(ic, ic + ic_layout.size());
    dofspan ic_residual{icbuf.data(), ic_layout};
    auto view = dof_view(res_mdg_h1);
    extract_icespan(ic_residual, view);
    io::PVDWriter<T, IDX, ndim> w{};
    w.data_directory = dir;
    w.collection_name = collection;
    w.register_fespace(space_h1);
    w.register_fields(res_mdg_h1, field_names(pb->pde));
    w.write_vtu(itime, (T)itime);
    return 0;
  });
}

}  // extern "C"
