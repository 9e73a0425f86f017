// Internal state of an iceicle_b200 context and the kernel launch interface.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/iceicle_b200.h"

namespace icx {

constexpr int MAX_P = 4;       // highest basis order with compiled kernels
constexpr int MAX_G = 2;       // highest geometry order with compiled kernels
constexpr int NFACE_GEO = 24;  // doubles per face quadrature point in the face geometry table

// field offsets of the face geometry table (structure of arrays: field f of
// point k at fgeo[f * nfq + k])
enum FaceGeoField {
  FG_N0 = 0, FG_N1 = 1, FG_WSQ = 2, FG_H = 3,
  FG_JIL = 4,   // 4 entries: Jinv of the left element, row-major [k][d]
  FG_HL = 8,    // 6 entries: transformation Hessian of the left element [m][ab], ab in {00,01,11}
  FG_JIR = 14,  // 4 entries
  FG_HR = 18    // 6 entries
};

// physical / discretization parameters passed by value to kernels
struct PhysParams {
  int pde;
  double mu, a[2], b[2];        // Burgers
  double mu_t;                  // Burgers viscosity along the second coordinate (mu; 0 in spacetime form)
  int spacetime;                // Burgers in (x, t): second coordinate is time (a[1] = 1, b[1] = 0, mu_t = 0)
  int st_connected;             // SPACETIME_PAST faces carry a past slab's trace in bvals (icx_spacetime_connect)
  double gamma, Pr, ns_mu;      // Navier-Stokes (unit reference parameters)
  double inv_gamma, inv_2gam2m1, mu_gamma_pr;  // 1/gamma, 1/(2(gamma^2-1)), mu*gamma/Pr
  int interior_penalty;
  double sigma_ic;
  double beta0, beta1;          // DDG coefficients (beta1 = 0 for interior penalty)
  int ns_flux;                  // Navier-Stokes convective flux: ICX_FLUX_VANLEER or ICX_FLUX_ROE
  // Navier-Stokes PDE-level boundaries (navier_stokes.hpp:976-1189): the
  // free stream of the characteristic (Riemann) boundary as density,
  // velocity and temperature, the gas constant of the equation of state,
  // and whether WALL_GENERAL is the no-slip isothermal wall (viscous) or the
  // slip wall (inviscid); wall temperatures per bcflag go into the boundary
  // data table at setup
  double fs_rho, fs_u[2], fs_T;
  double Rgas;
  int ns_viscous_wall;
  // Navier-Stokes viscosity law: 0 constant (ns_mu); 1 dimensionless
  // Sutherland mu(T) = suth[0] (T / suth[1])^1.5 (suth[1] + suth[2]) / (T + suth[2])
  int ns_visc;
  double suth[3];
};

// launch shapes of the tunable kernels (0: the compiled default). Every
// choice computes the same values in the same order: the tuner only moves
// work between threads, warps and CTAs.
struct TileChoice {
  int face_minb = 0;     // face_flux_kernel: CTAs per SM its register bound is compiled for
  int vol_threads = 0;   // vol_lift_kernel: threads per CTA (128 or 256; elements per CTA follow)
  int vol_minb = 0;      // vol_lift_kernel: CTAs per SM of its register bound
  int flow_rows[2] = {0, 0};  // data-flow ILU apply [FP64, FP32]: block rows per warp task
  int flow_ctas[2] = {0, 0};  // data-flow ILU apply: CTAs per SM of the persistent grid
  int flow_sched[2] = {0, 0}; // data-flow ILU apply: 1 completion counters, 2 sentinel values
};

// the data-flow ILU apply's schedule when a TileChoice leaves it at 0: the
// sentinel schedule (NS p=2, 256 x 256: 1.75 ms per FP64 apply against 2.41 ms
// with completion counters)
constexpr int kFlowSchedDefault = 2;
inline bool flow_sentinel(const TileChoice& t, int pi) {
  return (t.flow_sched[pi] ? t.flow_sched[pi] : kFlowSchedDefault) == 2;
}
// schedules 3, 4 and 5: the apply on element tiles / groups with one CTA
// per group (la_ilu_apply_groups), 4 with the matrix rows staged in shared
// memory, 5 with one lane per row and the group's vectors in shared memory,
// each where it fits; when the factors are tiled or grouped the default is
// 5 for FP32 factors (pi = 1) and 4 for FP64 ones (whose rows of 16-byte
// pairs need twice the registers)
inline int group_sched_default(int pi) { return pi == 1 ? 5 : 4; }
inline int ilu_schedule(const TileChoice& t, int pi, bool grouped) {
  const int sc = t.flow_sched[pi] ? t.flow_sched[pi] : (grouped ? group_sched_default(pi) : kFlowSchedDefault);
  return (sc >= 3 && !grouped) ? kFlowSchedDefault : sc;
}

// compiled volume tiles: threads per CTA and the resident CTAs per SM of the
// register bound (64 registers for the first and third, 80 for the others);
// the first is the default
struct VolTile {
  int threads, minb;
};
constexpr int kNumVolTiles = 4;
constexpr VolTile kVolTiles[kNumVolTiles] = {{256, 4}, {256, 3}, {128, 8}, {128, 6}};
// compiled rows per task of the data-flow ILU apply (0 in a TileChoice: the
// block size's default)
constexpr int kNumFlowRows = 4;
constexpr int kFlowRows[kNumFlowRows] = {2, 4, 6, 8};
// face_flux_kernel's default resident CTAs per SM; the tiles compiled beside
// it are one below and one above
int face_minb_default(int pde, bool ddg);
// the data-flow apply's default rows per task for a block size, and whether
// `rows` (0: the default) is compiled for it
int flow_rows_default(int bs);
bool flow_rows_compiled(int bs, int rows);

// device tables of one context (all device pointers)
struct DeviceMesh {
  TileChoice tile;
  int E = 0, F = 0, Fi = 0, Fb = 0, n_nodes = 0;
  int P = 0, G = 0, nb = 0, neq = 0, ng = 0, nq1 = 0, nqv = 0, nqf = 0;
  double* coord = nullptr;     // [n_nodes][2]
  int* el_nodes = nullptr;     // [E][ng]
  int* face_info = nullptr;    // [F][8]: elemL, elemR, fnl, fnr, orient, bctype, bcflag, boundary index
  int* el_face = nullptr;      // [E][4] face index per local face
  int* el_side = nullptr;      // [E][4] 0: element is L of that face, 1: R
  int* el_fso = nullptr;       // [E][4] face index * 4 + side + 2 * orientation (orientation of the R side, else 0)
  double* el_par = nullptr;    // batch of independent problems: [E][5] Burgers mu, a0, a1, b0, b1 per element (else null)
  double* vgeo = nullptr;      // [5][E*nqv]: Jinv00, Jinv01, Jinv10, Jinv11, w*detJ (clamped)
  double* fgeo = nullptr;      // [NFACE_GEO][F*nqf]
  double* tab_vol = nullptr;   // [nqv][nb][3]: phi, dphi/dxi0, dphi/dxi1
  double* tab_face = nullptr;  // [4 faces][2 orient][nqf][nb][6]: phi, d0, d1, h00, h01, h11
  double* tab_1d = nullptr;    // [2][nq1][p+1]: 1D Lagrange values, then derivatives, at the 1D Gauss points
  double* tab_fphi = nullptr;  // [4 faces][2 orient][nqf][nb]: phi of tab_face, compact
  // 1D factors of tab_face: [4 faces][p+1][3] value, d, d2 along the face's
  // fixed reference direction (lf & 1) at its constant coordinate, then
  // [4 faces][2 orient][nqf][p+1][3] along the varying direction
  double* tab_f1d = nullptr;
  double* tab_gvol = nullptr;  // [nqv][ng][2]: geometry basis gradients at volume points
  double* tab_gface = nullptr; // [4][2][nqf][ng][6]: geometry basis phi, d0, d1, h00, h01, h11 at face points
  double* tab_gcen = nullptr;  // [ng]: geometry basis at the element centroid
  double* qw_face = nullptr;   // [nqf]
  double* bvals = nullptr;     // [Fb*nqf][neq] Dirichlet or Neumann data at boundary points
  double* src = nullptr;       // [E*nqv][neq] source at volume points (or null)
  double* face_flux = nullptr; // scratch [F*nqf][neq]: (f_visc - f_adv) * w * sqrt(g)
  double* face_grad = nullptr; // scratch [F][2][nqf][neq][2]: interface-correction terms (sigma_ic != 0)
  int* bsr_rowptr = nullptr;   // [E+1]
  int* bsr_colidx = nullptr;   // [nnzb]
  int* bsr_diag = nullptr;     // [E] position of the diagonal block
  int* face_blk = nullptr;     // [F][4] block positions: LL, LR, RL, RR (-1 if none)
  int nnzb = 0;
};

}  // namespace icx

struct icx_ctx {
  int device = 0;
  std::string err;
  // mesh (host)
  bool has_mesh = false, has_space = false, has_disc = false, ready = false;
  int nx = 0, ny = 0, geo_order = 1;
  double xmin[2] = {0, 0}, xmax[2] = {1, 1};
  int bctype[4] = {0, 0, 0, 0}, bcflag[4] = {0, 0, 0, 0};
  std::vector<double> coord;                  // [n_nodes][2]
  std::vector<int> el_nodes;                  // [E][ng]
  std::vector<int> faces;                     // [F][7] reference face order
  int n_interior = 0;
  int n_elem = 0;                             // elements (nx * ny for one grid)
  std::vector<int> el_level;                  // [E] anti-diagonal index i + j of the element in its grid
  std::vector<int> el_i, el_j, el_grid;       // [E] grid position (i, j) of the element and its grid's index
  int ilu_tile = 0;                           // block-ILU(0) on s x s element tiles (0: the whole grid)
  std::vector<int> ilu_groups;                // block-ILU(0) per element group (set: overrides ilu_tile)
  int ilu_plan_gen = 1;                       // changes whenever the tiling or the groups change
  // a batch of independent problems (icx_batch_create): the parts it was
  // built from (not owned) and each element's Burgers coefficients (mu, a0, a1, b0, b1)
  std::vector<icx_ctx*> parts;
  std::vector<double> el_par;
  int p = 0;
  int basis = ICX_BASIS_LAGRANGE;             // solution basis family
  icx::PhysParams phys{};
  int conv_flux = 0;
  std::vector<double> wall_T;                 // Navier-Stokes isothermal wall temperature per bcflag
  std::vector<icx_point_fn> dirichlet_fn, neumann_fn;
  std::vector<void*> dirichlet_user, neumann_user;
  icx_point_fn source_fn = nullptr;
  void* source_user = nullptr;
  icx::DeviceMesh dm;
  // solver scratch (device), grown on demand
  std::vector<void*> scratch;
  struct icx_solver_work* sw = nullptr;  // Newton / GMRES buffers (icx_solver.cu)
  struct icx_mdg_state* mdg = nullptr;   // MDG-ICE selection and Jacobian pattern (icx_mdg.cu)
  struct icx_explicit_work* ew = nullptr; // explicit time-stepping buffers (icx_explicit.cu)
  struct icx_lpc* lpc = nullptr;          // learned block preconditioner model (attached, not owned)
  struct icx_lpc_work* lpcw = nullptr;    // its per-context buffers (icx_lpc.cu)
  struct icx_host_pipe* hp = nullptr;     // streams and staging buffers of icx_form_residuals_host (icx_pipeline.cu)
};

namespace icx {
// kernels (icx_residual.cu)
cudaError_t launch_geometry(const DeviceMesh& dm, cudaStream_t s);
// `mid` (optional) is recorded on s between the face and volume kernels
cudaError_t launch_residual(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                            cudaStream_t s, cudaEvent_t mid = nullptr);
// the volume (domain integral) contributions alone, faces left out
cudaError_t launch_residual_domain(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                                   cudaStream_t s);
// Jacobian (icx_jacobian.cu)
cudaError_t launch_jacobian_fd(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                               double* vals, double eps, cudaStream_t s);
// FP64 residual, FP32-quadrature FD Jacobian (FP32 values, eps = sqrt(FLT_EPSILON))
cudaError_t launch_jacobian_fd_f32(const DeviceMesh& dm, const PhysParams& pp, const double* u, double* res,
                                   float* vals, cudaStream_t s);
cudaError_t launch_bsr_spmv(const DeviceMesh& dm, const double* vals, const double* x, double* y,
                            cudaStream_t s);
// the same with FP32 values and FP32 accumulation (x, y FP64)
cudaError_t launch_bsr_spmv_f32(const DeviceMesh& dm, const float* vals, const double* x, double* y,
                                cudaStream_t s);
// releases the Newton / GMRES buffers of a context (icx_solver.cu)
void free_solver_work(icx_ctx* c);
// releases the MDG-ICE state of a context (icx_mdg.cu)
void free_mdg(icx_ctx* c);
// re-evaluates boundary/source data at the current host coordinates, uploads
// them and recomputes the geometry factors (icx_host.cu)
icx_status refresh_geometry(icx_ctx* c);
// values of the pn+1 equispaced Lagrange polynomials of [-1, 1] at x (icx_host.cu)
void lagrange_values(int pn, double x, double* N);
// the same with first derivatives
void lagrange_values_derivs(int pn, double x, double* N, double* dN);
// values of the pn+1 one-dimensional functions of a basis family (ICX_BASIS_*) at x
void basis_values(int kind, int pn, double x, double* N);
// releases the explicit time-stepping buffers of a context (icx_explicit.cu)
void free_explicit(icx_ctx* c);
// Gauss-Legendre points in the reference order (+x1, -x1, ..., 0) and weights (icx_host.cu)
void gauss_legendre_points(int n, double* x, double* w);
// physical point of reference point xi in element e (geometry transformation, icx_host.cu)
void element_point(const icx_ctx* c, int e, const double xi[2], double x[2]);
// learned block preconditioner (icx_lpc.cu): features and correction from the
// FP64 Jacobian, the correction z = (I + C) y, and the release of its buffers
cudaError_t lpc_build(icx_ctx* c, const double* vals, cudaStream_t s);
cudaError_t lpc_apply(icx_ctx* c, const double* y, double* z, cudaStream_t s);
// the attached model's output layer is all zero (its correction C = 0)
bool lpc_zero_correction(const icx_ctx* c);
void free_lpc_work(icx_ctx* c);
// releases the host-pipeline streams and buffers (icx_pipeline.cu)
void free_host_pipe(icx_ctx* c);
// solver internals the training uses (icx_solver.cu): copy a Jacobian into the
// solver and build preconditioner `kind` with mixed-precision copies; apply it;
// the FP32 copy of the Jacobian
// (sweeps < 0 keeps the solver's Jacobi sweeps per triangle)
icx_status solver_prepare_pc(icx_ctx* c, const double* vals, int kind, int sweeps);
cudaError_t solver_apply_pc(icx_ctx* c, int kind, bool mixed, const double* x, double* z, cudaStream_t s);
const float* solver_vals32(icx_ctx* c);
// one block-ILU(0) apply on the data-flow schedule (factors from
// solver_prepare_pc with kind 2), and the apply's error flag (read, then
// cleared with the completion counters when set)
cudaError_t solver_apply_ilu_flow(icx_ctx* c, bool mixed, const double* x, double* z, cudaStream_t s);
icx_status solver_take_pc_err(icx_ctx* c, int* err);
// the per-group pieces of a batch of independent solves (icx_pset.cu):
// buffers and options, the FP64 residual with the Jacobian (precision 2: FP32
// quadrature), the preconditioner, the Jacobian as operator, the factorisation
// flag, whether the preconditioner apply can be captured in a graph, and the
// reference's line searches (1 Wolfe, 2 Corrigan, else the full step)
icx_status solver_group_ready(icx_ctx* c, int precision, int pc_sweeps, int ilu_tile, bool graphs);
cudaError_t solver_linearise(icx_ctx* c, const double* u, double* res, int precision, cudaStream_t s);
cudaError_t solver_build_pc(icx_ctx* c, int kind, bool mixed, cudaStream_t s);
cudaError_t solver_operator(icx_ctx* c, bool mixed, const double* x, double* y, cudaStream_t s);
const int* solver_flag(icx_ctx* c);
bool solver_graphable(icx_ctx* c, int pc, bool mixed);
unsigned long long solver_graph_key(icx_ctx* c, int pc, bool mixed);
double solver_line_search(int kind, const std::function<double(double)>& f, const icx_newton_options& o);
}  // namespace icx
