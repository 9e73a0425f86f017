/*
 * iceicle_b200: B200-native DG residual / FD-Jacobian / Newton path behind a C ABI.
 *
 * Every entry point returns an icx_status (0 = ICX_OK). Pointers named d_* are
 * device pointers (CUDA global memory of the context's device); everything else
 * is host memory. Calls taking a `stream` (a cudaStream_t passed as void*, NULL
 * = legacy default stream) are stream-ordered and do not synchronise.
 *
 * Reference interfaces replaced (paths relative to the reference project root):
 *   CL = src/FiniteElement/include/iceicle/disc/conservation_law.hpp
 *   ME = src/FiniteElement/include/iceicle/mesh/mesh.hpp
 *   FS = src/FiniteElement/include/iceicle/fespace/fespace.hpp
 *   FR = src/solvers/include/iceicle/form_residual.hpp
 *   FJ = src/solvers/include/iceicle/form_petsc_jacobian.hpp
 *   PN = src/solvers/include/iceicle/petsc_newton.hpp
 *   NU = src/solvers/include/iceicle/nonlinear_solver_utils.hpp
 */
#ifndef ICEICLE_B200_H
#define ICEICLE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int icx_status;
#define ICX_OK 0
#define ICX_ERR_INVALID 1       /* bad argument or call order */
#define ICX_ERR_CUDA 2          /* a CUDA runtime call failed */
#define ICX_ERR_UNSUPPORTED 3   /* configuration outside what the kernels implement */
#define ICX_ERR_NONFINITE 4     /* non-finite residual norm */
#define ICX_ERR_NOT_CONVERGED 5 /* nonlinear or linear iteration limit reached */
#define ICX_ERR_NOMEM 6         /* device allocation failed */
#define ICX_ERR_SIZE 7          /* problem size beyond a fixed capacity */
#define ICX_ERR_NO_DEVICE 8     /* no CUDA device (no CPU fallback exists) */

/* boundary condition kinds: the reference BOUNDARY_CONDITIONS values
 * (src/FiniteElement/include/iceicle/geometry/face.hpp:23-90) */
#define ICX_BC_PERIODIC 0
#define ICX_BC_NEUMANN 2
#define ICX_BC_DIRICHLET 3
#define ICX_BC_EXTRAPOLATION 4
/* Navier-Stokes PDE-level kinds (navier_stokes.hpp:976-1189; the Burgers
 * fluxes implement none, so such faces contribute nothing there) */
#define ICX_BC_RIEMANN 5            /* characteristic far field against the free stream */
#define ICX_BC_NO_SLIP_ISOTHERMAL 6 /* wall at rest at the temperature of its bcflag */
#define ICX_BC_SLIP_WALL 7          /* inviscid wall: momentum mirrored */
#define ICX_BC_WALL_GENERAL 8       /* no-slip isothermal when viscous (mu > 0), else slip */
#define ICX_BC_SPACETIME_PAST 11
#define ICX_BC_SPACETIME_FUTURE 12
#define ICX_BC_INTERIOR 13

#define ICX_BASIS_LAGRANGE 0 /* FESPACE_ENUMS::LAGRANGE: equispaced nodal tensor-product basis */
#define ICX_BASIS_LEGENDRE 1 /* FESPACE_ENUMS::LEGENDRE: tensor products of Legendre polynomials */
#define ICX_PDE_BURGERS 0
#define ICX_PDE_NAVIER_STOKES 1
#define ICX_FLUX_UPWIND 0  /* BurgersUpwind (burgers.hpp:114-170) */
#define ICX_FLUX_VANLEER 1 /* navier_stokes::VanLeer (navier_stokes.hpp:776-864) */
#define ICX_FLUX_ROE 2     /* Roe's approximate Riemann solver with Harten's entropy fix (no reference
                              counterpart: the reference's Navier-Stokes has only Van Leer) */

/* host callback x[2] -> out[neq]: the reference's std::function<void(const T*, T*)>
 * dirichlet_callbacks / neumann_callbacks / user_source (CL:145-160) */
typedef void (*icx_point_fn)(const double* x, double* out, void* user);

typedef struct icx_ctx icx_ctx;

typedef struct icx_layout_info {
  int n_elem;         /* E */
  int nbasis;         /* basis functions per element, (p+1)^2 */
  int neq;            /* equations per basis function */
  int block_size;     /* nbasis * neq: the BSR block edge */
  long long n_dof;    /* E * block_size: length of u and res */
  int n_faces, n_interior_faces;
  int n_nodes;        /* geometry nodes */
  int nnz_blocks;     /* blocks of the Jacobian pattern */
  int nq_vol, nq_face;/* quadrature points per element / per face */
} icx_layout_info;

/* ---- context ---------------------------------------------------------- */
icx_status icx_create(icx_ctx** out, int device);
void icx_destroy(icx_ctx* ctx);
const char* icx_last_error(const icx_ctx* ctx);

/* ---- mesh: AbstractMesh uniform hypercube constructor (ME:553-913) ------
 * nelem[2], xmin[2], xmax[2]; bctypes/bcflags indexed left, bottom, right, top
 * (the reference's face-number convention). Node lattice is x fastest. */
icx_status icx_mesh_uniform(icx_ctx* ctx, int ndim, const int* nelem, const double* xmin, const double* xmax,
                            int geo_order, const int* bctypes, const int* bcflags);
/* overwrite node coordinates (host, n_nodes x 2); the reference writes
 * mesh.coord then calls update_coord_els (ME:994-999) */
icx_status icx_mesh_set_coords(icx_ctx* ctx, const double* xy);
icx_status icx_mesh_get_coords(const icx_ctx* ctx, double* xy);
/* element node lists [E][(g+1)^2] and faces [F][7] = (elemL, elemR, face_nr_l,
 * face_nr_r, orientation_r, bctype, bcflag) in the reference's face order */
icx_status icx_mesh_topology(const icx_ctx* ctx, int* conn, int* faces, int* n_interior);

/* ---- FESpace (FS:200-416): tensor-product Lagrange, Gauss-Legendre ------ */
icx_status icx_fespace(icx_ctx* ctx, int basis_order);
/* FESpace{mesh, basis, GAUSS_LEGENDRE, p} with basis ICX_BASIS_LAGRANGE or
 * ICX_BASIS_LEGENDRE (HypercubeLegendreBasis, basis/legendre.hpp:282-327:
 * u = sum c_ij P_i(xi0) P_j(xi1), index i * (p+1) + j, unnormalised Legendre
 * polynomials); icx_basis_node_coords refuses the modal Legendre basis */
icx_status icx_fespace_basis(icx_ctx* ctx, int basis_order, int basis);

/* ---- ConservationLawDDG (CL:92-218) ------------------------------------ */
icx_status icx_disc_burgers(icx_ctx* ctx, double mu, const double* a, const double* b);
/* SpacetimeBurgersFlux / SpacetimeBurgersUpwind / SpacetimeBurgersDiffusion
 * (disc/burgers.hpp:261-474) with BurgersCoefficients<T, 1>{mu, a, b}: the
 * second mesh coordinate is time, F = ((a + b u / 2) u - mu du/dx, u), the
 * upwind flux includes the time normal, and there is no diffusion along time.
 * Boundaries: ICX_BC_SPACETIME_FUTURE (top of a slab) extrapolates; a
 * SPACETIME_PAST face (bottom of a slab, value 11) without a connected past
 * slab contributes nothing, as in the reference's discretization without
 * spacetime information; sigma_ic is ignored (no homogeneity tensor). */
icx_status icx_disc_spacetime_burgers(icx_ctx* ctx, double mu, double a, double b);
/* SpacetimeConnection (disc/SpacetimeConnection.hpp:102-189) for a slab on top
 * of a solved one: the past slab's solution d_u_past (device, `past`'s
 * layout) is evaluated at the quadrature points of ctx's SPACETIME_PAST faces
 * (located on the past slab's SPACETIME_FUTURE elements by their x
 * coordinate), and those faces then take it as exterior state: time-upwind
 * convective flux from the past trace, and DDG diffusion with it as the
 * neighbour value, which vanishes on an interface at constant t (the only
 * kind accepted). Both contexts must be set-up spacetime Burgers slabs whose
 * interface lies at the same t. The connection holds until ctx's mesh or
 * boundary data are recomputed (icx_setup, icx_mesh_set_coords); call it
 * again after those. */
icx_status icx_spacetime_connect(icx_ctx* ctx, const icx_ctx* past, const double* d_u_past);
icx_status icx_disc_navier_stokes(icx_ctx* ctx, double gamma, double Pr, double mu, int conv_flux);
/* data of the Navier-Stokes PDE-level boundaries (Physics::isothermal_temperatures
 * and Physics::free_stream, navier_stokes.hpp:679-682): wall temperatures
 * indexed by the faces' bcflag (n_walls <= 8), the free stream's density,
 * velocity magnitude, unit direction and temperature, and the gas constant
 * of the ideal-gas equation of state (EoS::Rgas, default 287.052874). The
 * temperature unit is the equation of state's: p = rho Rgas T with unit
 * reference parameters. */
icx_status icx_disc_ns_boundary(icx_ctx* ctx, const double* wall_temperatures, int n_walls, double rho_inf,
                                double u_inf, const double u_direction[2], double T_inf, double Rgas);
/* the Navier-Stokes viscosity law (Physics' viscosity function,
 * navier_stokes.hpp:218-287): kind 0 constant_viscosity (the mu given to
 * icx_disc_navier_stokes, which also resets to it); kind 1
 * DimensionlessSutherlands, mu(T) = mu_ratio (T / T0_ratio)^1.5
 * (T0_ratio + Ts_ratio) / (T + Ts_ratio) at the state's temperature, with the
 * ratios of its members (mu_0 / ref.mu, T_0 / ref.T, T_s / ref.T); the flux
 * is then the full (viscous) Navier-Stokes flux. */
icx_status icx_disc_ns_viscosity(icx_ctx* ctx, int kind, double mu_ratio, double T0_ratio, double Ts_ratio);
/* public members interior_penalty and sigma_ic (CL:137-143) */
icx_status icx_disc_options(icx_ctx* ctx, int interior_penalty, double sigma_ic);
icx_status icx_disc_dirichlet(icx_ctx* ctx, int bcflag, icx_point_fn fn, void* user);
icx_status icx_disc_neumann(icx_ctx* ctx, int bcflag, icx_point_fn fn, void* user);
icx_status icx_disc_source(icx_ctx* ctx, icx_point_fn fn, void* user);

/* Builds device tables (geometry factors, quadrature tabulations, boundary and
 * source data evaluated through the callbacks). Must follow the calls above;
 * icx_mesh_set_coords after it re-runs the geometry and callback tabulation. */
icx_status icx_setup(icx_ctx* ctx);
icx_status icx_get_layout(const icx_ctx* ctx, icx_layout_info* info);

/* ---- hot path ------------------------------------------------------------
 * form_residual(fespace, disc, u, res) (FR:56-268): d_res = R(d_u), both of
 * length n_dof in the reference layout u[(elem*nbasis + idof)*neq + ieq]. */
icx_status icx_form_residual(icx_ctx* ctx, const double* d_u, double* d_res, void* stream);

/* Allocation-free variant of icx_form_residual (no counterpart in the
 * reference, which has no device code). For callers that cannot allocate
 * device memory while they evaluate residuals: a host framework that owns all
 * device memory through its own pool and forbids other allocations during a
 * solve, or a time-critical loop that must not pay the device-wide
 * synchronisation of cudaMalloc/cudaFree. It calls no allocating routine; the
 * face-flux scratch lives in a fixed 8 MiB __device__ array per device, so it
 * serves problems with n_faces * nq_face * neq <= 2^20 (the 128x128 p=3
 * Navier-Stokes mesh needs 660,480) and returns ICX_ERR_SIZE beyond that.
 * The first call on a device looks up the array's address (make it before
 * any stream capture on that device). All calls on a device share the array:
 * calls that overlap on the GPU race and must be serialised by the caller. */
icx_status icx_form_residual_noalloc(icx_ctx* ctx, const double* d_u, double* d_res, void* stream);

/* form_residual (FR:56-268) for n_states states in host memory: h_u and h_res
 * hold n_states vectors of n_dof doubles each (page-locked host memory lets
 * the copies run asynchronously). The copy of state k+1 to the device, the
 * kernels of state k and the copy of residual k-1 to the host overlap; the
 * call returns when every residual is in h_res. *elapsed_ms (may be NULL)
 * is the device time from the first copy to the last, by CUDA events. Uses
 * the context's residual scratch: no other residual call on this context may
 * run at the same time. */
icx_status icx_form_residuals_host(icx_ctx* ctx, int n_states, const double* h_u, double* h_res,
                                   double* elapsed_ms);
/* diagnostics: the same computation as icx_form_residual, with CUDA events
 * around each kernel on `stream`; synchronises and returns the two kernel
 * durations in milliseconds (face fluxes, volume + face lifting). */
icx_status icx_form_residual_timed(icx_ctx* ctx, const double* d_u, double* d_res, void* stream,
                                   double* ms_face, double* ms_volume);

/* Jacobian block pattern: rows = elements; per row the element itself and its
 * face neighbours in ascending element order. rowptr[E+1], colidx[nnz_blocks]. */
icx_status icx_jacobian_pattern(const icx_ctx* ctx, int* rowptr, int* colidx);

/* form_petsc_jacobian_fd (FJ:55-317) straight into BSR: d_vals holds
 * nnz_blocks dense row-major block_size^2 blocks in the pattern above;
 * also writes d_res = R(d_u). eps <= 0 selects sqrt(machine epsilon). */
icx_status icx_form_jacobian_fd(icx_ctx* ctx, const double* d_u, double* d_res, double* d_vals, double eps,
                                void* stream);

/* The same Jacobian with the flux quadrature in FP32 (the FP32 build of
 * form_petsc_jacobian_fd, CMakeLists.txt:19-22 USE_SINGLE_PRECISION): states,
 * metrics, tabulations, fluxes and sums rounded to FP32, perturbations scaled
 * by sqrt(FLT_EPSILON), blocks written as FP32 into d_vals32; d_res = R(d_u)
 * in FP64. */
icx_status icx_form_jacobian_fd_f32(icx_ctx* ctx, const double* d_u, double* d_res, float* d_vals32, void* stream);

/* y = J x for the BSR Jacobian (PETSc MatMult on the AIJ matrix, PN:243) */
icx_status icx_bsr_spmv(icx_ctx* ctx, const double* d_vals, const double* d_x, double* d_y, void* stream);

/* ---- MDG-ICE (moving discontinuous Galerkin, interface condition enforcement)
 * icx_mdg_select: geo_dof_map over the given face indices, i.e. the nodes of
 * those faces become geometry unknowns (fe_function/geo_layouts.hpp:359-498);
 * hyper_rectangle != 0 applies mesh_parameterizations::hyper_rectangle
 * (geo_layouts.hpp:510-540): nodes on the box keep the coordinate they sit on
 * and slide along it. Geometry parameters x: per selected node its free
 * coordinates (extract_geospan / update_mesh, component_span.hpp:177-210). */
icx_status icx_mdg_select(icx_ctx* ctx, int ntraces, const int* traces, int hyper_rectangle);
icx_status icx_mdg_info(const icx_ctx* ctx, int* n_selected_nodes, int* n_geo);
icx_status icx_mdg_selected_nodes(const icx_ctx* ctx, int* nodes);
icx_status icx_mdg_get_x(const icx_ctx* ctx, double* x);        /* host */
icx_status icx_mdg_set_x(icx_ctx* ctx, const double* x);        /* host; moves the mesh */
/* form_mdg_residual (form_residual.hpp:335-381): d_ic[n_selected_nodes * neq] */
icx_status icx_form_mdg_residual(icx_ctx* ctx, const double* d_u, double* d_ic, void* stream);
/* form_residual(fespace, disc, geo_map, [u; x], [res; ic]) (form_residual.hpp:426-452);
 * x (host) may be NULL to keep the current mesh */
icx_status icx_form_residual_mdg(icx_ctx* ctx, const double* d_u, const double* x, double* d_res, double* d_ic,
                                 void* stream);
/* CSR pattern of the Jacobian of [res; ic] w.r.t. [u; x]: nrow = n_dof + n_ic,
 * ncol = n_dof + n_geo; rowptr/colidx (host) may be NULL to query sizes */
icx_status icx_mdg_jacobian_pattern(icx_ctx* ctx, long long* nrow, long long* ncol, long long* nnz, int* rowptr,
                                    int* colidx);
/* form_petsc_jacobian_fd + form_petsc_mdg_jacobian_fd (form_petsc_jacobian.hpp:55-317, 665-1049):
 * [res; ic] and the CSR values of the full Jacobian at the current mesh */
icx_status icx_form_jacobian_mdg_fd(icx_ctx* ctx, const double* d_u, double* d_res, double* d_ic,
                                    double* d_csr_vals, double eps, void* stream);

/* ---- regularised Gauss-Newton / Levenberg-Marquardt for MDG-ICE
 * (CorriganLM::solve, src/solvers/include/iceicle/corrigan_lm.hpp:363-717) with
 * the matrix-free subproblem (J^T J + D) p = J^T r, D = lambda_u |J_col| on the
 * PDE unknowns and max(lambda_b, lambda_b |J_col|) on the geometry unknowns
 * (corrigan_lm.hpp:68-109), solved by GMRES without preconditioner. */
typedef struct icx_lm_options {
  double tau_abs, tau_rel;
  int kmax;
  double lambda_u, lambda_b;
  int linesearch;            /* 0 none, 2 corrigan (nonlinear_solver_utils.hpp:173-191, 236-257) */
  int ls_max_it;
  double ls_alpha_initial, ls_alpha_max, ls_alpha_min;
  int gmres_restart, gmres_max_it;
  double gmres_rtol;
  int max_rejections;        /* bound on rejected steps in a row */
  int verbosity;
  /* 1: form the subproblem matrix (explicitly_form_subproblem = true,
   * corrigan_lm.hpp:426-530): J^T J + diag(lambda_u |J_col|, lambda_b |J_col|)
   * + lambda_lag |r| K^T K on the isoparametric continuous space + the
   * element-wise regularisation lambda_el of elements that inverted, solved
   * by GMRES with its ILU(0) (PCILU). 0 (default): the matrix-free
   * J^T J + diag(lambda_u |J_col|, max(lambda_b, lambda_b |J_col|)) operator
   * without preconditioner (the MATSHELL path, corrigan_lm.hpp:68-109). */
  int explicit_subproblem;
  double lambda_lag;         /* CorriganLM::lambda_lag (default 1e-5) */
  /* 1: return after the first subproblem solve (the KSPSolve of the first
   * iteration) with its solution p in place of the unknowns: d_u <- p_u,
   * x <- p_x; nothing is updated. 0 (default): the solve. */
  int step_only;
} icx_lm_options;

typedef struct icx_lm_report {
  int iterations, converged, rejections;
  double r0, r_final;
  int linear_iterations_total;
  double residual_history[64];
  double alpha_history[64];
  double linear_relres_max;  /* the largest relative residual a subproblem solve ended with */
} icx_lm_report;

icx_status icx_lm_default_options(icx_lm_options* opt);
/* d_u (device) and the geometry parameters x (host, n_geo) are updated in place */
icx_status icx_lm_solve(icx_ctx* ctx, double* d_u, double* x, const icx_lm_options* opt, icx_lm_report* rep);

/* ---- Newton solver (PetscNewton, PN:37-337; ConvergenceCriteria, NU:24-60) */
typedef struct icx_newton_options {
  double tau_abs, tau_rel;
  int kmax;
  int linesearch;          /* 0 none, 1 wolfe (NU:207-233), 2 corrigan (NU:236-257) */
  int ls_max_it;
  double ls_alpha_initial, ls_alpha_max, ls_alpha_min, ls_c1, ls_c2;
  int gmres_restart;       /* GMRES(m) restart length */
  int gmres_max_it;        /* total inner iterations per Newton step */
  double gmres_rtol;       /* relative tolerance of the linear solve */
  int preconditioner;      /* 0 none, 1 block-Jacobi, 2 block-ILU0, 3 two-step block-Jacobi
                              G (2 I - J G), 4 block-ILU0 factors with Jacobi-sweep triangular solves,
                              5 learned: (I + C) times preconditioner 4, or times 2 when pc_sweeps = 0
                              (icx_lpc_attach); a step whose linear solve misses gmres_rtol with 3-5
                              is solved again with 2. A model whose output layer is all zero (C = 0)
                              makes 5 its base exactly: the solve is then 2 (or 4), fallback rule included */
  int verbosity;
  /* 0: all FP64. 1: mixed - the linear solves read FP32 copies of the
   * Jacobian (SpMV) and of the preconditioner (block inverses / ILU factors,
   * formed in FP64 then rounded) with FP32 accumulation, and keep the GMRES
   * Krylov basis in FP32 (its inner products and updates accumulate in
   * FP64); the Hessenberg and Givens rotations, the solution update, the
   * Newton residual, its norm and the line search stay FP64, so the converged
   * state is judged in FP64.
   * 2: as 1, with the Jacobian's flux quadrature itself in FP32
   * (icx_form_jacobian_fd_f32); the preconditioner is factored in FP64 from
   * those FP32 values. Newton is then FP64 iterative refinement around FP32
   * linearisations: its residual, norm, line search and update stay FP64.
   * 3: as 1, with the block-ILU(0) factors of a tiled or grouped
   * preconditioner (ilu_tile, icx_set_ilu_groups) stored in BF16 and widened
   * to FP32 in the apply (the one-lane-per-row form, ilu_sched 5; where its
   * shared memory does not fit, and on whole-grid factors, the FP32 copies
   * of 1). The preconditioner only changes GMRES iterations: the converged
   * state is judged in FP64 as in 1. */
  int precision;
  /* preconditioner 4 (block-ILU(0) factors applied by Jacobi sweeps): the
   * sweeps per triangular solve */
  int pc_sweeps;
  /* 1 (default): replay each GMRES Arnoldi step (preconditioner, operator,
   * both Gram-Schmidt passes, norm, normalisation and the copy of the
   * reductions) as one CUDA graph once it has run eagerly, for preconditioners
   * 0-4 (block-ILU(0) on its default sentinel schedule). The same kernels run
   * in the same order: results are identical with 0. */
  int cuda_graphs;
  /* block-ILU(0) on ilu_tile x ilu_tile element tiles for preconditioners 2,
   * 4 and 5: blocks that couple two tiles are dropped, which is block-Jacobi
   * over the tiles with ILU(0) inside each (PETSc's parallel default,
   * PCBJACOBI with PCILU sub-solves, petsc_newton.hpp:179-182, one block per
   * tile). 0 (default): ILU(0) over the whole grid in natural order, the
   * single-process PCILU. Negative: keep the context's setting
   * (icx_set_ilu_tile). Changes the preconditioner and so the GMRES
   * iterations, not the converged state. */
  int ilu_tile;
  /* 1: the GMRES operator is the directional difference of the FP64
   * residual, J v ~ (R(u + h v) - R(u)) / h with h = sqrt(DBL_EPSILON)
   * (sqrt(n) + |u|) / |v| (the matrix-free products of icx_mfnk_solve); the
   * assembled FD Jacobian then serves the preconditioner only (PETSc's
   * -snes_mf_operator). One residual evaluation per Krylov step instead of
   * the BSR product, in every precision mode. 0 (default): the assembled
   * Jacobian's BSR product. */
  int matrix_free;
  /* GMRES orthogonalisation: 1 (default) classical Gram-Schmidt with a
   * second pass every Arnoldi step; 0 one pass, which is PETSc's default
   * (KSPGMRES with refinement "never", what the reference's
   * KSPSetFromOptions, petsc_newton.hpp:175-182, gets without options) and
   * reads the Krylov basis half as often */
  int gmres_cgs_refine;
} icx_newton_options;

typedef struct icx_newton_report {
  int iterations;
  int converged;
  double r0, r_final;
  int linear_iterations_total;
  double residual_history[64];
  double alpha_history[64];
  int pc_fallbacks;  /* steps whose linear solve was redone with block-ILU(0) (preconditioners 3-5: the
                        solve missed gmres_rtol, or stalled: under 10 % residual reduction over 20
                        restart cycles) */
  int linear_iterations[64]; /* GMRES iterations of each Newton step (fallback included) */
  int graph_steps;           /* Arnoldi steps replayed from CUDA graphs */
} icx_newton_report;

/* Linear solve J x = b with the BSR values d_vals (the KSPSolve of
 * petsc_newton.hpp:243-244): restarted right-preconditioned GMRES(restart),
 * preconditioner 0 none / 1 block-Jacobi / 2 block-ILU(0). Returns
 * ICX_ERR_NOT_CONVERGED when the relative residual stays above rtol. */
icx_status icx_gmres_solve(icx_ctx* ctx, const double* d_vals, const double* d_b, double* d_x, int restart,
                           int maxit, double rtol, int preconditioner, int* iterations, double* relres, void* stream);

/* y = M^-1 x for the block-ILU(0) preconditioner of the BSR matrix d_vals
 * (the factors icx_gmres_solve / icx_newton_solve build; precision 1: from
 * FP32 copies with FP32 accumulation; 2: tiled or grouped factors from BF16
 * copies in the one-lane-per-row apply with FP32 arithmetic, as Newton
 * precision 3, the FP32 copies where it does not fit). schedule 0 or 1: the data-flow apply
 * the solvers use; 2: the row-pipelined apply, one CTA per grid row
 * (ICX_ERR_UNSUPPORTED when the context is not one grid with the 5-point
 * element pattern; it is slower than the data-flow apply on the measured
 * workloads). The apply runs `repeat` times after one factorization;
 * *ms_per_apply (may be NULL) is its mean device time by CUDA events. */
/* the context's block-ILU(0) tiling used by icx_gmres_solve, icx_ilu_apply,
 * icx_krylov_samples and by icx_newton_solve when its ilu_tile < 0 (tile side
 * in elements, 0: the whole grid; see icx_newton_options.ilu_tile). No
 * reference counterpart: the reference selects the PC through PETSc options. */
icx_status icx_set_ilu_tile(icx_ctx* ctx, int tile);
int icx_get_ilu_tile(const icx_ctx* ctx);
/* block-ILU(0) per element group: groups[E] (NULL: back to the tiling) - the
 * blocks coupling two groups are dropped, e.g. a partitioned mesh's owned
 * elements in one group and each ghost row in its own, which is the
 * block-Jacobi across ranks of PETSc's parallel default (bjacobi + ilu)
 * (no reference counterpart as an entry point) */
icx_status icx_set_ilu_groups(icx_ctx* ctx, const int* groups);
/* the block-ILU(0) preconditioner alone (PCSetUp / PCApply of
 * petsc_newton.hpp:179-183): factor the BSR values d_vals (precision 1: also
 * its FP32 copies), then apply y = M^-1 x on a stream, any number of times */
icx_status icx_pc_factor(icx_ctx* ctx, const double* d_vals, int precision);
icx_status icx_pc_apply(icx_ctx* ctx, const double* d_x, double* d_y, int precision, void* stream);
icx_status icx_ilu_apply(icx_ctx* ctx, const double* d_vals, const double* d_x, double* d_y, int precision,
                         int schedule, int repeat, double* ms_per_apply);
icx_status icx_newton_default_options(icx_newton_options* opt);
icx_status icx_newton_solve(icx_ctx* ctx, double* d_u, const icx_newton_options* opt, icx_newton_report* rep);
/* MFNK (matrix_free_newton_krylov.hpp:62-365) without geometry unknowns:
 * Newton with the Jacobian applied matrix-free as
 * (R(u + eps p) - R(u)) / eps, eps = sqrt(machine epsilon), GMRES without
 * preconditioner (opt->preconditioner is ignored), the line searches of
 * icx_newton_solve (non-finite trial residuals count as 1e100) and the
 * stopping test |R| <= tau_abs after every step, as the reference's solver
 * applies it. rep->iterations = Newton steps taken. */
icx_status icx_mfnk_solve(icx_ctx* ctx, double* d_u, const icx_newton_options* opt, icx_newton_report* rep);

/* ---- explicit time stepping (ExplicitEuler explicit_euler.hpp:30-181,
 * RK3TVD tvd_rk3.hpp:30-277, RK3SSP ssp_rk3.hpp:30-241; FixedTimestep,
 * CFLTimestep, TimestepTermination, TfinalTermination explicit_utils.hpp:60-180).
 * The update is u += dt M^-1 R(u) per element with M the element mass matrix.
 * RK3SSP evaluates all three stage residuals at the step's initial state, as
 * the reference's stage function does. The CFL timestep (Burgers only) uses
 * the running maximum of |a + b u / 2| over the volume points of every
 * residual evaluation of the solve, as BurgersFlux::lambda_max does. */
typedef struct icx_explicit_options {
  int scheme;       /* 0 ExplicitEuler, 1 RK3TVD, 2 RK3SSP */
  int timestep;     /* 0 FixedTimestep (dt), 1 CFLTimestep (cfl) */
  double dt, cfl;
  int termination;  /* 0 TimestepTermination (ntime), 1 TfinalTermination (tfinal) */
  int ntime;
  double tfinal;
} icx_explicit_options;

typedef struct icx_explicit_report {
  int steps;              /* itime at the end */
  double time;            /* time at the end */
  double dt_last;
  double lambda_max;      /* Burgers: the running maximum wave speed */
  int singular_elements;  /* elements whose mass matrix had no inverse (RK3TVD: 1e-8 r there) */
} icx_explicit_report;

icx_status icx_explicit_default_options(icx_explicit_options* opt);
/* d_u (device) advanced in place */
icx_status icx_explicit_solve(icx_ctx* ctx, double* d_u, const icx_explicit_options* opt, icx_explicit_report* rep);
/* d_out = M^-1 d_r element by element and equation by equation */
icx_status icx_mass_inverse_apply(icx_ctx* ctx, const double* d_r, double* d_out, void* stream);

/* ---- batches of independent problems (no counterpart in the reference, which
 * solves one problem per process). icx_batch_create lays the meshes of n_parts
 * set-up contexts side by side in one new context: every call above then
 * works on all parts at once (one launch per kernel), with each part's
 * discretization unchanged. Parts must share the PDE, basis order, geometry
 * order, interior_penalty / sigma_ic and (Navier-Stokes) the fluid constants;
 * Burgers coefficients, mesh sizes, coordinates and boundary data may differ.
 * The parts must outlive the batch. u / res of the batch are the parts' vectors
 * concatenated in part order; icx_batch_offsets gives each part's first
 * element (n_parts + 1 entries). Not available on a batch: MDG-ICE, the CFL
 * timestep. A Newton solve on a batch uses one line search and one stopping
 * test for the concatenated residual. */
icx_status icx_batch_create(icx_ctx** out, int device, int n_parts, icx_ctx* const* parts);
icx_status icx_batch_offsets(const icx_ctx* batch, int* elem_offsets);

/* ---- sets of independent problems of uneven mesh size and basis order (no
 * counterpart in the reference). icx_pset_create groups n_parts set-up
 * contexts by basis order into batches (icx_batch_create's rules hold within
 * an order; every part has the same PDE). The set's vectors hold each order's
 * parts side by side, orders ascending, parts in their given order within an
 * order; icx_pset_offsets gives part k's first unknown (offsets[k], in the
 * caller's part numbering; the part's own n_dof unknowns follow) and
 * offsets[n_parts] = the total. The parts must outlive the set.
 * icx_pset_newton_solve runs one Newton solve per part, each on its own
 * (petsc_newton.hpp:205-329): its own residual norm and stopping test, its own
 * GMRES Krylov space, Hessenberg matrix and convergence, its own line search
 * and step length. A Newton iteration of the set launches each kernel once
 * per basis order for all parts; each GMRES Arnoldi step of the whole set is
 * one CUDA graph launch (cuda_graphs = 1, preconditioners whose apply is
 * graph-invariant). reports[k] is part k's report; the status is
 * ICX_ERR_NOT_CONVERGED when a part did not converge. Preconditioners 0-2 and
 * 4; precision 0-2 as icx_newton_solve. */
typedef struct icx_pset icx_pset;
typedef struct icx_pset_stats {
  int newton_rounds;       /* Newton iterations of the set (the slowest part's) */
  int arnoldi_steps;       /* Arnoldi steps of the set (each covers every part still iterating) */
  int graph_launches;      /* of those, replayed from CUDA graphs */
  int line_search_rounds;  /* residual evaluations of the whole set for the line searches */
  int orders;              /* basis-order groups */
} icx_pset_stats;
icx_status icx_pset_create(icx_pset** out, int device, int n_parts, icx_ctx* const* parts);
void icx_pset_destroy(icx_pset* set);
icx_status icx_pset_offsets(const icx_pset* set, long long* offsets);
/* every part's residual R(u_k) into d_res (the set's layout) */
icx_status icx_pset_residual(icx_pset* set, const double* d_u, double* d_res);
icx_status icx_pset_newton_solve(icx_pset* set, double* d_u, const icx_newton_options* opt,
                                 icx_newton_report* reports, icx_pset_stats* stats);
const char* icx_pset_last_error(const icx_pset* set);

/* Krylov samples for training the learned preconditioner: the GMRES solve of
 * icx_gmres_solve (from a zero guess, FP64) that also copies the true residual
 * at every restart and every `every`-th Arnoldi vector into d_samples
 * ([capacity][n_dof], device) until it is full; *n_samples = copies made. */
icx_status icx_krylov_samples(icx_ctx* ctx, const double* d_vals, const double* d_b, double* d_x, int restart, int maxit,
                              double rtol, int preconditioner, int every, int capacity, double* d_samples,
                              int* n_samples, int* iterations, double* relres);

/* ---- learned block preconditioner (no counterpart in the reference): an MLP
 * from each normalised Jacobian diagonal block J_ee / |J_ee|_F (bs x bs values)
 * through two ReLU layers of `hidden` units to a bs x bs correction C_e; the
 * Newton preconditioner 5 applies z = (I + C) y with y the block-ILU(0)
 * factors applied by pc_sweeps Jacobi sweeps per triangle. BF16 products on
 * the tensor cores with FP32 accumulation; FP32 master weights. */
/* BF16 GEMM on the tensor cores (tcgen05.mma, TMEM accumulator, TMA operand
 * loads): C = A . B^T with A [M][lda] and B [N][ldb] row-major BF16 (device),
 * FP32 accumulation; optional bias [N] and ReLU, output FP32 (C32 [M][ldc])
 * and/or BF16 (C16 [M][ldc16]); accumulate = 1 adds into C32 atomically and
 * allows splits > 1 (split-K). K, lda, ldb multiples of 8, lda, ldb >= K,
 * A and B 16-byte aligned. The kernel of the learned preconditioner's MLP
 * (no reference counterpart), exported for tests. Synchronises the stream. */
icx_status icx_gemm_bf16_nt(int M, int N, int K, const void* d_A, int lda, const void* d_B, int ldb,
                            const float* d_bias, int relu, float* d_C32, int ldc, void* d_C16, int ldc16,
                            int accumulate, int splits, void* stream);

typedef struct icx_lpc icx_lpc;
typedef struct icx_lpc_train_options {
  int steps;               /* Adam steps on this Jacobian */
  int batch;               /* residual samples per step */
  int random;              /* of which this many are seeded Gaussian vectors instead of Krylov samples */
  int sweeps;              /* Jacobi sweeps per triangle of the preconditioner being trained (0: exact ILU(0)) */
  double lr;               /* Adam step size */
  unsigned long long seed; /* sample selection */
} icx_lpc_train_options;
typedef struct icx_lpc_train_report {
  int steps;
  double loss_first, loss_last; /* mean of |r - J z(r)|^2 / |r|^2 over the step's samples */
  double loss_history[64];
} icx_lpc_train_report;
icx_status icx_lpc_create(icx_lpc** out, int device, int block_size, int hidden, unsigned long long seed);
void icx_lpc_destroy(icx_lpc* model);
icx_status icx_lpc_info(const icx_lpc* model, int* block_size, int* hidden, long long* n_params, long long* steps);
/* FP32 parameters W1 [hidden][bs^2], b1, W2 [hidden][2 hidden], b2, W3 [bs^2][hidden], b3 (host arrays) */
icx_status icx_lpc_get_params(const icx_lpc* model, float* params);
icx_status icx_lpc_set_params(icx_lpc* model, const float* params);
/* use `model` (NULL: detach) for preconditioner 5 of this context; the model must outlive the attachment */
icx_status icx_lpc_attach(icx_ctx* ctx, icx_lpc* model);
/* the correction C ([n_elem][bs][bs] FP32, device; may be NULL) of the attached model for Jacobian d_vals */
icx_status icx_lpc_forward(icx_ctx* ctx, const double* d_vals, float* d_corr);
/* Adam steps of the attached model on Jacobian d_vals (FP64 BSR) and residual
 * samples d_samples ([n_samples][n_dof], device) */
icx_status icx_lpc_train(icx_ctx* ctx, const double* d_vals, int n_samples, const double* d_samples,
                         const icx_lpc_train_options* opt, icx_lpc_train_report* rep);
/* held-out check of the attached model on Jacobian d_vals and residual
 * samples r: with y the base preconditioner's output (block-ILU(0) FP32
 * factors; `sweeps` Jacobi sweeps per triangle, 0: exact solves),
 * a = r - J y and b = J C y, sums[0..2] = the sums over the samples of
 * <a, b> / |r|^2, |b|^2 / |r|^2 and |a|^2 / |r|^2. The training loss of
 * z = (I + g C) y is then sums[2] - 2 g sums[0] + g^2 sums[1]. */
icx_status icx_lpc_calibrate(icx_ctx* ctx, const double* d_vals, int n_samples, const double* d_samples, int sweeps,
                             double sums[3]);

/* ---- restart files and VTU output (host files; d_u and d_ic are device
 * arrays). Not available on a batch. */
/* write_restart (fe_function/restart.hpp:20-59): writes <dir>/restart<k>_<rank>
 * (dir NULL: "RESTART" under the working directory, created if missing): the
 * node coordinates "x y " per node, a newline, then u in layout order, each
 * value followed by a space, 16 significant digits. */
icx_status icx_write_restart(icx_ctx* ctx, const double* d_u, int k, int rank, const char* dir);
/* read_restart (restart.hpp:68-108): reads <dir>/<name>_<rank>, moves the mesh
 * nodes to the stored coordinates (as icx_mesh_set_coords) and fills d_u.
 * ICX_ERR_INVALID when the file is missing or holds too few numbers (the
 * reference leaves such values unread). */
icx_status icx_read_restart(icx_ctx* ctx, double* d_u, const char* name, int rank, const char* dir);

#define ICX_VTU_SOLUTION 0 /* PVDWriter::register_fields(u, field_names) */
#define ICX_VTU_RESIDUAL 1 /* PVDWriter::register_residuals(u, residual_names, disc) */
/* PVDWriter::write_vtu(itime, time) (io/pvd_writer.hpp:1095-1140): writes
 * <dir>/<collection><itime>.vtu (dir NULL: "iceicle_data"; collection NULL:
 * "data", or "residuals" for ICX_VTU_RESIDUAL as the reference's driver names
 * it) in the discontinuous layout, values with `precision` significant digits
 * (the reference prints 8). ICX_VTU_SOLUTION writes the fields of d_u;
 * ICX_VTU_RESIDUAL the residual of d_u, then its domain-integral part
 * ("domain_" prefix) and its face part ("trace_" prefix). names: neq names,
 * or NULL for the reference's ("u" / "residual" for Burgers; "rho", "rhou",
 * "rhov", "rhoe" / "density_conservation", "momentum_u_conservation",
 * "momentum_v_conservation", "energy_conservation" for Navier-Stokes). */
icx_status icx_write_vtu(icx_ctx* ctx, const double* d_u, int kind, int itime, const char* dir,
                         const char* collection, const char* const* names, int precision);
/* the MDG interface-conservation residual d_ic ([selected node][neq], the tail
 * of icx_form_residual_mdg's output) as the reference's implicit driver writes
 * it (solvers_lua_interface.hpp:589-632): scattered to the mesh nodes (zero at
 * unselected nodes) and written over the isoparametric H1 space; collection
 * NULL: "mdg_residuals"; names NULL: the field names above. */
icx_status icx_write_vtu_mdg(icx_ctx* ctx, const double* d_ic, int itime, const char* dir, const char* collection,
                             const char* const* names, int precision);

/* ---- workload callbacks (icx_point_fn) ------------------------------------
 * icx_wl_constant: user -> double[1 + n] = {n, v_0 .. v_{n-1}}: out = v
 * icx_wl_sine_product: user -> double[1] = {amp}: out[0] = amp sin(2 pi x) sin(2 pi y)
 * icx_wl_ns_mms_state / icx_wl_ns_mms_source: user -> double[7] =
 *   {gamma, Pr, mu, p_inf, A, u0, v0}: manufactured Navier-Stokes state
 *   (conservative variables) and the matching source term */
void icx_wl_constant(const double* x, double* out, void* user);
void icx_wl_sine_product(const double* x, double* out, void* user);
/* user -> double[4] = {x0, slope, u_left, u_right}: out[0] = u_left if x < x0 + slope*y else u_right */
void icx_wl_oblique_step(const double* x, double* out, void* user);
void icx_wl_ns_mms_state(const double* x, double* out, void* user);
void icx_wl_ns_mms_source(const double* x, double* out, void* user);

/* physical coordinates of the Lagrange nodes of every element, [E][nbasis][2]
 * (for nodal initial states, as the reference's nodal interpolation) */
icx_status icx_basis_node_coords(const icx_ctx* ctx, double* xy);

/* ---- launch-shape autotuner (no counterpart in the reference, whose kernels
 * are CPU loops). The tunable kernels are compiled in several launch shapes
 * that compute the same values in the same order, so a choice changes speed,
 * never results. 0 in any field selects the compiled default.
 *   face_minb   face flux kernel: resident CTAs per SM of its register bound,
 *               the default D or D - 1 / D + 1 (D = 5; 3 for Navier-Stokes
 *               with the DDG flux)
 *   vol_threads, vol_minb   volume + lifting kernel: (256, 4) default,
 *               (256, 3), (128, 8), (128, 6) (elements per CTA = threads /
 *               volume points)
 *   ilu_rows[k], ilu_ctas[k]   data-flow block-ILU(0) apply, k = 0 FP64 and
 *               1 FP32 factors: block rows per warp task (2, 4, 6, 8; at most
 *               the block size and 24 register values per lane), CTAs per
 *               SM of the persistent grid (1 to 4; capped by occupancy) and the
 *               schedule: 1 completion counters per element, 2 outputs
 *               pre-filled with a sentinel and polled directly (the default
 *               on whole-grid factors), 3 on tiled or grouped factors one CTA
 *               per tile running the tile's levels between CTA barriers, 4 the
 *               same with each warp's next task rows copied ahead into shared
 *               memory, 5 one lane per matrix row with the tile's vectors in
 *               shared memory (the defaults there: 5 for FP32 factors, 4 for
 *               FP64 ones; each falls back to the one
 *               below where its shared memory does not fit; 3 to 5 are 2 on
 *               whole-grid factors; 5 sums each row's columns in order, so
 *               its results differ from the others' in rounding); for 3 to 5
 *               ilu_ctas picks the threads per CTA instead: 0 the default
 *               (256 FP64, 512 FP32 factors), 1 / 2 / 3 512 / 256 / 128 */
typedef struct icx_tile_choice {
  int face_minb;
  int vol_threads, vol_minb;
  int ilu_rows[2];
  int ilu_ctas[2];
  int ilu_sched[2];
} icx_tile_choice;

typedef struct icx_tune_report {
  icx_tile_choice chosen;      /* the context's choice after the call */
  int from_cache;              /* bit set per part (ICX_TUNE_*) taken from the process-wide cache untimed */
  int n_timed;                 /* candidates timed */
  int n_rejected;              /* candidates whose output was not bit-identical to the default's (never chosen) */
  double residual_ms_default;  /* face + volume kernels, device time per residual (L2 flushed before each) */
  double residual_ms_tuned;
  double ilu_ms_default[2];    /* one block-ILU(0) apply, [FP64, FP32] */
  double ilu_ms_tuned[2];
} icx_tune_report;

#define ICX_TUNE_RESIDUAL 1 /* face and volume kernels, timed at d_u */
#define ICX_TUNE_ILU 2      /* data-flow ILU apply with FP64 factors of the FD Jacobian at d_u */
#define ICX_TUNE_ILU_FP32 4 /* the same with FP32 factors */
#define ICX_TUNE_RETIME 8   /* time even when the cache holds a choice for the key */

/* Times every compiled shape of the selected kernels on this context's mesh
 * at the state d_u (device, not modified), checks each output against the
 * default shape's bit for bit, and keeps the fastest in the context. Choices
 * are cached per process under the key (dimension, basis order p, equations
 * neq, geometry order, viscous flux) and reused untimed by later contexts with
 * the same key unless ICX_TUNE_RETIME is set. rep may be NULL. */
icx_status icx_autotune(icx_ctx* ctx, const double* d_u, int parts, icx_tune_report* rep);
icx_status icx_tile_get(const icx_ctx* ctx, icx_tile_choice* tile);
/* ICX_ERR_INVALID for a shape that is not compiled for this context. icx_setup
 * returns a context to the default shapes (call icx_autotune again after it;
 * the cached choice then costs nothing). */
icx_status icx_tile_set(icx_ctx* ctx, const icx_tile_choice* tile);

#ifdef __cplusplus
}
#endif
#endif
