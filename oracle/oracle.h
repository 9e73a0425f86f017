/*
 * CPU oracle for the DG residual / FD-Jacobian path: a plain-C restatement of
 * the reference algorithm (iceicle's ConservationLawDDG with the Burgers and
 * compressible Navier-Stokes fluxes, form_residual and form_petsc_jacobian_fd)
 * used ONLY as the checker in tests, in smoke() and as the CPU baseline in
 * bench.py. Nothing in the product links, imports or calls it.
 *
 * Parity of this restatement is pinned against the reference's own headers
 * compiled here (oracle/ref_harness, built into oracle/_ref).
 */
#ifndef ICEICLE_ORACLE_H
#define ICEICLE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* host callback for boundary data and sources: x[2] -> out[neq] */
typedef void (*orc_point_fn)(const double* x, double* out, void* user);

/* problem description; same layout as the reference harness' ref_problem */
typedef struct orc_problem {
  int pde;              /* 0: Burgers, 1: Navier-Stokes */
  int nx, ny;           /* elements per direction */
  int geo_order;        /* geometry (node) order of the quads */
  int p;                /* Lagrange basis order */
  double xmin[2], xmax[2];
  int bctype[4];        /* BOUNDARY_CONDITIONS values: left, bottom, right, top */
  int bcflag[4];
  int interior_penalty;
  double sigma_ic;
  double mu;            /* Burgers viscosity */
  double a[2], b[2];    /* Burgers linear / nonlinear advection */
  double gamma, Pr;     /* Navier-Stokes */
  double ns_mu;         /* constant viscosity */
  int n_dirichlet;
  orc_point_fn dirichlet[8];
  void* dirichlet_user[8];
  int n_neumann;
  orc_point_fn neumann[8];
  void* neumann_user[8];
  orc_point_fn source;
  void* source_user;
  int spacetime;        /* Burgers in (x, t): SpacetimeBurgersFlux/Upwind/Diffusion, no diffusion along t */
  int basis;            /* solution basis: 0 Lagrange (equispaced nodes), 1 Legendre */
  /* Navier-Stokes: convective flux (0 or 1 Van Leer, 2 Roe) and the data of
   * the PDE-level boundaries (Physics::isothermal_temperatures and
   * Physics::free_stream, navier_stokes.hpp:679-682) */
  int ns_flux;
  int n_wall;
  double wall_T[8];
  double fs_rho, fs_u_inf, fs_dir[2], fs_T;
  /* viscosity law: 0 constant_viscosity{ns_mu}; 1 DimensionlessSutherlands
   * with suth = {mu_ratio, T_0_ratio, T_s_ratio} (navier_stokes.hpp:260-287) */
  int ns_visc;
  double suth[3];
} orc_problem;

/* reference BOUNDARY_CONDITIONS enumerators used here */
enum {
  ORC_BC_PERIODIC = 0, ORC_BC_PARALLEL_COM = 1, ORC_BC_NEUMANN = 2, ORC_BC_DIRICHLET = 3,
  ORC_BC_EXTRAPOLATION = 4, ORC_BC_RIEMANN = 5, ORC_BC_NO_SLIP_ISOTHERMAL = 6, ORC_BC_SLIP_WALL = 7,
  ORC_BC_WALL_GENERAL = 8, ORC_BC_SPACETIME_PAST = 11, ORC_BC_SPACETIME_FUTURE = 12, ORC_BC_INTERIOR = 13
};

int orc_n_nodes(const orc_problem* pb);
int orc_n_faces(const orc_problem* pb);
int orc_neq(const orc_problem* pb);
/* equispaced node lattice, x fastest */
void orc_mesh_coords(const orc_problem* pb, double* coord);
/* element node lists and faces (elemL, elemR, face_nr_l, face_nr_r, orient, bctype, bcflag) */
int orc_mesh_topology(const orc_problem* pb, int* conn, int* faces, int* n_interior);
/* res = R(u); returns 0 on success */
int orc_form_residual(const orc_problem* pb, const double* coord, const double* u, double* res);
/* FD Jacobian (reference perturbation scheme) into block-sparse rows: block
 * row e holds the diagonal block and one block per face neighbour, columns in
 * ascending element order; rowptr[E+1], colidx[nnzb], vals[nnzb*bs*bs]
 * (each block row-major). Also writes res. */
int orc_bsr_pattern(const orc_problem* pb, int* rowptr, int* colidx);
int orc_form_jacobian_fd(const orc_problem* pb, const double* coord, const double* u, double* res,
                         const int* rowptr, const int* colidx, double* vals);

/* MDG-ICE over the selected traces, optionally with the hyper_rectangle
 * boundary parametrisation. orc_mdg_select returns the number of geometry
 * parameters and writes the selected nodes and x (extract_geospan). */
int orc_mdg_select(const orc_problem* pb, const double* coord, int ntr, const int* traces, int hyper, int* nsel,
                   int* sel_nodes, double* x);
/* [res; ic] at [u; x] */
int orc_mdg_residual(const orc_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                     const double* u_and_x, double* res_and_ic);
/* dense (N + nsel*neq) x (N + ngeo) Jacobian of [res; ic] w.r.t. [u; x]; writes [res; ic] */
int orc_mdg_jacobian_dense(const orc_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                           const double* u, const double* x, double* res_and_ic, double* J);

/* physical coordinates of the Lagrange basis nodes [E][nb][2] (basis index
 * dim 0 slowest); -1 for a modal basis */
int orc_basis_node_coords(const orc_problem* pb, const double* coord, double* xy);

/* workload point callbacks (oracle/workloads.c; same meaning as the product's
 * icx_wl_* exports, derived separately) */
void orc_wl_constant(const double* x, double* out, void* user);
void orc_wl_sine_product(const double* x, double* out, void* user);
void orc_wl_oblique_step(const double* x, double* out, void* user);
void orc_wl_ns_mms_state(const double* x, double* out, void* user);
void orc_wl_ns_mms_source(const double* x, double* out, void* user);

/* pointwise fluxes (consistency tests): convective numerical flux of the
 * problem's PDE, physical flux F[eq][2] at state u with gradient g[eq][2],
 * and the exterior state of a Navier-Stokes PDE-level boundary */
void orc_numerical_flux(const orc_problem* pb, const double* uL, const double* uR, const double* n, double* f);
void orc_physical_flux(const orc_problem* pb, const double* u, const double* g, double* F);
void orc_ns_boundary_state(const orc_problem* pb, const double* uL, const double* n, int bctype, int bcflag,
                           double* uR);

/* the same Jacobian as (row, col, value) triplets whose duplicates add;
 * returns the number of triplets (written up to cap), -1 on failure */
long long orc_mdg_jacobian_coo(const orc_problem* pb, const double* coord, int ntr, const int* traces, int hyper,
                               const double* u, const double* x, double* res_and_ic, long long cap, int* rows,
                               int* cols, double* vals);

/* per-element stiffness of the isoparametric continuous space [E][ng][ng]
 * and per-element minimum of det J over the volume quadrature points [E]
 * (the regularisation inputs of the explicitly formed LM subproblem) */
int orc_cg_stiffness(const orc_problem* pb, const double* coord, double* K);
int orc_min_detj(const orc_problem* pb, const double* coord, double* mins);

/* selected nodes sel[nsel] and parameter offsets cols[nsel + 1] of an MDG
 * selection; returns nsel */
int orc_mdg_layout(const orc_problem* pb, const double* coord, int ntr, const int* traces, int hyper, int* sel,
                   int* cols);

/* element mass matrices [E][nb][nb] (finite_element.hpp:587-610) */
int orc_mass_matrices(const orc_problem* pb, const double* coord, double* M);
/* explicit time stepping: scheme 0 Euler, 1 TVD-RK3, 2 SSP-RK3; dt_kind 0
 * fixed, 1 CFL; term_kind 0 ntime steps, 1 tfinal (explicit_*.hpp, ssp_rk3.hpp,
 * tvd_rk3.hpp, explicit_utils.hpp); u updated in place */
int orc_explicit_solve(const orc_problem* pb, const double* coord, double* u, int scheme, int dt_kind, double dt_fixed,
                       double cfl, int term_kind, int ntime, double tfinal, int* steps_out, double* time_out);

#ifdef __cplusplus
}
#endif
#endif
