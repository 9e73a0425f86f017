// Explicit time stepping around the GPU residual, restating the reference's
// explicit solvers (src/solvers/include/iceicle/):
//   ExplicitEuler  explicit_euler.hpp:88-137   u += dt M^-1 R(u)
//   RK3TVD         tvd_rk3.hpp:108-233         Shu-Osher three-stage form,
//                  u <- alfa u_old + beta u + beta dt M^-1 R(u) per stage
//   RK3SSP         ssp_rk3.hpp:107-187         three stages whose residuals the
//                  reference evaluates at the step's initial state (its stage
//                  lambda reads the outer u), then u += dt/6 r1 + dt/6 r2 + 2dt/3 r3
// with FixedTimestep / CFLTimestep and TimestepTermination / TfinalTermination
// (explicit_utils.hpp:69-180). M is the element mass matrix
// sum_q phi_i phi_j w det J with det J not clamped (calculate_mass_matrix,
// finite_element.hpp:587-610), inverted once per solve per element in shared
// memory. The CFL wave speed is the reference's BurgersFlux::lambda_max: the
// running maximum of |a + b u / 2| over every volume point of every residual
// evaluation since the solve began (burgers.hpp:65-108).
#include <cmath>
#include <cstring>
#include <vector>

#include "icx_internal.h"
#include "icx_blockinv.cuh"
#include "icx_linalg.h"

struct icx_explicit_work {
  long long n = 0;
  int E = 0, nb = 0;
  double* minv = nullptr;  // [E][nb][nb]
  int* singular = nullptr; // [E]
  double* r = nullptr;     // residual
  double* d1 = nullptr;    // M^-1 r of the stages
  double* d2 = nullptr;
  double* d3 = nullptr;
  double* uold = nullptr;
  unsigned long long* lam = nullptr;  // running max |lambda|: bits of a non-negative double
};

namespace icx {

template <int NB, int G>
__global__ void __launch_bounds__(256) mass_inverse_kernel(DeviceMesh dm, double* __restrict__ minv,
                                                           int* __restrict__ singular) {
  constexpr int NG = (G + 1) * (G + 1);
  extern __shared__ double sh[];
  double* a = sh;                 // NB x NB
  double* fcol = a + NB * NB;     // NB
  double* sw = fcol + NB;         // [nqv] weights
  double* sdet = sw + dm.nqv;     // [nqv] det J
  int* perm = reinterpret_cast<int*>(sdet + dm.nqv);
  int* colsrc = perm + NB;
  __shared__ int s_sing;
  const int e = blockIdx.x;
  const int nqv = dm.nqv;
  for (int q = threadIdx.x; q < nqv; q += blockDim.x) {
    double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
    for (int n = 0; n < NG; ++n) {
      int gn = dm.el_nodes[e * NG + n];
      double x0 = dm.coord[2 * gn], x1 = dm.coord[2 * gn + 1];
      double d0 = dm.tab_gvol[(q * NG + n) * 2], d1 = dm.tab_gvol[(q * NG + n) * 2 + 1];
      J00 += d0 * x0; J01 += d1 * x0;
      J10 += d0 * x1; J11 += d1 * x1;
    }
    sdet[q] = J00 * J11 - J01 * J10;
    sw[q] = dm.tab_vol[(size_t)nqv * NB * 3 + q];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
    int i = t / NB, j = t - i * NB;
    double m = 0.0;
    for (int q = 0; q < nqv; ++q)
      m += dm.tab_vol[((size_t)q * NB + i) * 3] * dm.tab_vol[((size_t)q * NB + j) * 3] * sw[q] * sdet[q];
    a[t] = m;
  }
  __syncthreads();
  gj_invert<NB>(a, perm, fcol, &s_sing);
  __syncthreads();
  if (threadIdx.x == 0) singular[e] = s_sing;
  write_inverse<NB>(a, perm, colsrc, s_sing, minv + (size_t)e * NB * NB);
}

// d[e][i][k] = sum_j Minv[e][i][j] r[e][j][k]; a singular element gives
// 1e-8 r (the fallback of tvd_rk3.hpp:185-199; other schemes refuse singular
// mass matrices before stepping)
__global__ void mass_apply_kernel(int E, int nb, int neq, const double* __restrict__ minv,
                                  const int* __restrict__ singular, const double* __restrict__ r,
                                  double* __restrict__ d) {
  const long long n = (long long)E * nb * neq;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t / (nb * neq));
    const int rem = (int)(t - (long long)e * nb * neq);
    const int i = rem / neq, k = rem - i * neq;
    const double* re = r + (size_t)e * nb * neq;
    if (singular[e]) {
      d[t] = 1e-8 * re[i * neq + k];
      continue;
    }
    const double* m = minv + ((size_t)e * nb + i) * nb;
    double acc = 0.0;
    for (int j = 0; j < nb; ++j) acc += m[j] * re[j * neq + k];
    d[t] = acc;
  }
}

// u += c1 d1 (+ c2 d2 + c3 d3, applied in that order)
__global__ void explicit_update_kernel(long long n, double* __restrict__ u, double c1, const double* __restrict__ d1,
                                       double c2, const double* __restrict__ d2, double c3,
                                       const double* __restrict__ d3) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = u[i] + c1 * d1[i];
    if (d2) v = v + c2 * d2[i];
    if (d3) v = v + c3 * d3[i];
    u[i] = v;
  }
}

// one TVD stage: u = alfa u_old + beta u, then u += (beta dt) d
__global__ void tvd_stage_kernel(long long n, double* __restrict__ u, const double* __restrict__ uold, double alfa,
                                 double beta, double bdt, const double* __restrict__ d) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = alfa * uold[i] + beta * u[i];
    u[i] = v + bdt * d[i];
  }
}

// Burgers wave speed |a + b u / 2| at every volume point; running maximum
__global__ void burgers_lambda_kernel(DeviceMesh dm, PhysParams pp, const double* __restrict__ u,
                                      unsigned long long* lam) {
  const long long npt = (long long)dm.E * dm.nqv;
  double best = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < npt; t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t / dm.nqv), q = (int)(t - (long long)e * dm.nqv);
    double uq = 0.0;
    for (int i = 0; i < dm.nb; ++i) uq += u[(size_t)e * dm.nb + i] * dm.tab_vol[((size_t)q * dm.nb + i) * 3];
    const double* pa = dm.el_par ? dm.el_par + 5 * (size_t)e + 1 : pp.a;
    const double* pb = dm.el_par ? dm.el_par + 5 * (size_t)e + 3 : pp.b;
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      double l = pa[d] + 0.5 * pb[d] * uq;
      s += l * l;
    }
    best = fmax(best, sqrt(s));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(lam, (unsigned long long)__double_as_longlong(best));
}

static unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (unsigned)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

void free_explicit(icx_ctx* c) {
  if (!c || !c->ew) return;
  icx_explicit_work* w = c->ew;
  void* ptrs[] = {w->minv, w->singular, w->r, w->d1, w->d2, w->d3, w->uold, w->lam};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete w;
  c->ew = nullptr;
}

}  // namespace icx

namespace {

icx_status xerr(icx_ctx* c, icx_status st, const std::string& m) {
  if (c) c->err = m;
  return st;
}

#define XCK(expr)                                                                                          \
  do {                                                                                                     \
    cudaError_t _e = (expr);                                                                               \
    if (_e != cudaSuccess) return xerr(c, ICX_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

icx_status ensure_explicit(icx_ctx* c) {
  const icx::DeviceMesh& dm = c->dm;
  long long n = (long long)dm.E * dm.nb * dm.neq;
  if (c->ew && c->ew->n == n && c->ew->E == dm.E && c->ew->nb == dm.nb) return ICX_OK;
  icx::free_explicit(c);
  icx_explicit_work* w = c->ew = new icx_explicit_work();
  w->n = n;
  w->E = dm.E;
  w->nb = dm.nb;
  XCK(cudaMalloc((void**)&w->minv, sizeof(double) * (size_t)dm.E * dm.nb * dm.nb));
  XCK(cudaMalloc((void**)&w->singular, sizeof(int) * dm.E));
  double** vecs[] = {&w->r, &w->d1, &w->d2, &w->d3, &w->uold};
  for (double** p : vecs) XCK(cudaMalloc((void**)p, sizeof(double) * n));
  XCK(cudaMalloc((void**)&w->lam, sizeof(unsigned long long)));
  return ICX_OK;
}

// inverse element mass matrices at the current mesh; *n_singular elements had none
icx_status build_mass_inverse(icx_ctx* c, cudaStream_t s, int* n_singular) {
  const icx::DeviceMesh& dm = c->dm;
  icx_explicit_work* w = c->ew;
  cudaError_t e = cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * (dm.nb * dm.nb + dm.nb + 2 * dm.nqv) + sizeof(int) * 2 * dm.nb;
#define ICX_MASS_CASE(NBV, GV)                                                                     \
  if (dm.nb == NBV && dm.G == GV) {                                                                 \
    icx::mass_inverse_kernel<NBV, GV><<<dm.E, 256, smem, s>>>(dm, w->minv, w->singular);            \
    e = cudaGetLastError();                                                                         \
  }
  ICX_MASS_CASE(4, 1) ICX_MASS_CASE(9, 1) ICX_MASS_CASE(16, 1) ICX_MASS_CASE(25, 1)
  ICX_MASS_CASE(4, 2) ICX_MASS_CASE(9, 2) ICX_MASS_CASE(16, 2) ICX_MASS_CASE(25, 2)
#undef ICX_MASS_CASE
  XCK(e);
  std::vector<int> sing(dm.E);
  XCK(cudaMemcpyAsync(sing.data(), w->singular, sizeof(int) * dm.E, cudaMemcpyDeviceToHost, s));
  XCK(cudaStreamSynchronize(s));
  int ns = 0;
  for (int v : sing) ns += v != 0;
  *n_singular = ns;
  return ICX_OK;
}

}  // namespace

extern "C" {

icx_status icx_explicit_default_options(icx_explicit_options* o) {
  if (!o) return ICX_ERR_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->scheme = 1;         // RK3TVD
  o->timestep = 0;       // FixedTimestep
  o->dt = 1e-3;
  o->cfl = 0.3;          // CFLTimestep default (explicit_utils.hpp:73)
  o->termination = 0;    // TimestepTermination
  o->ntime = 1;
  o->tfinal = 1.0;       // TfinalTermination default (explicit_utils.hpp:148)
  return ICX_OK;
}

icx_status icx_mass_inverse_apply(icx_ctx* c, const double* d_r, double* d_out, void* stream) {
  if (!c || !c->ready) return xerr(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_r || !d_out) return xerr(c, ICX_ERR_INVALID, "null device pointer");
  cudaStream_t s = (cudaStream_t)stream;
  icx_status st = ensure_explicit(c);
  if (st != ICX_OK) return st;
  int ns = 0;
  if ((st = build_mass_inverse(c, s, &ns)) != ICX_OK) return st;
  if (ns) return xerr(c, ICX_ERR_NONFINITE, "singular element mass matrix");
  const icx::DeviceMesh& dm = c->dm;
  icx::mass_apply_kernel<<<icx::grid_for(c->ew->n), 256, 0, s>>>(dm.E, dm.nb, dm.neq, c->ew->minv, c->ew->singular, d_r,
                                                                 d_out);
  XCK(cudaGetLastError());
  return ICX_OK;
}

icx_status icx_explicit_solve(icx_ctx* c, double* d_u, const icx_explicit_options* o, icx_explicit_report* rep) {
  if (!c || !c->ready) return xerr(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !o) return xerr(c, ICX_ERR_INVALID, "null argument");
  if (o->scheme < 0 || o->scheme > 2 || o->timestep < 0 || o->timestep > 1 || o->termination < 0 ||
      o->termination > 1)
    return xerr(c, ICX_ERR_INVALID, "scheme 0..2, timestep 0..1, termination 0..1");
  if (o->timestep == 1 && c->phys.pde != ICX_PDE_BURGERS)
    return xerr(c, ICX_ERR_UNSUPPORTED, "the CFL timestep needs the flux's wave speed (Burgers)");
  if (o->timestep == 1 && !c->parts.empty())
    return xerr(c, ICX_ERR_UNSUPPORTED, "a batch has one timestep per problem: use a fixed timestep");
  const cudaStream_t s = 0;
  icx_status st = ensure_explicit(c);
  if (st != ICX_OK) return st;
  icx_explicit_work* w = c->ew;
  const icx::DeviceMesh& dm = c->dm;
  const long long n = w->n;
  int ns = 0;
  if ((st = build_mass_inverse(c, s, &ns)) != ICX_OK) return st;
  if (ns && o->scheme != 1) return xerr(c, ICX_ERR_NONFINITE, "singular element mass matrix");
  // CFL reference length: min over elements of det(J at the reference centroid)^(1/2)
  double reflen = 1e8;
  if (o->timestep == 1) {
    const int g = c->geo_order, g1 = g + 1, ng = g1 * g1;
    double N[16], dN[16];
    icx::lagrange_values_derivs(g, 0.0, N, dN);
    for (int e = 0; e < dm.E; ++e) {
      double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
      for (int a = 0; a < g1; ++a)
        for (int b = 0; b < g1; ++b) {
          int gn = c->el_nodes[(size_t)e * ng + a * g1 + b];
          double d0 = dN[a] * N[b], d1 = N[a] * dN[b];
          double x0 = c->coord[2 * gn], x1 = c->coord[2 * gn + 1];
          J00 += d0 * x0; J01 += d1 * x0;
          J10 += d0 * x1; J11 += d1 * x1;
        }
      double r = std::pow(J00 * J11 - J01 * J10, 1.0 / 2);
      reflen = std::min(reflen, r);
    }
  }
  XCK(cudaMemsetAsync(w->lam, 0, sizeof(unsigned long long), s));
  const bool burgers = c->phys.pde == ICX_PDE_BURGERS;
  auto residual = [&](const double* u) -> cudaError_t {
    cudaError_t e = icx::launch_residual(dm, c->phys, u, w->r, s);
    if (e == cudaSuccess && burgers) {
      icx::burgers_lambda_kernel<<<icx::grid_for((long long)dm.E * dm.nqv), 256, 0, s>>>(dm, c->phys, u, w->lam);
      e = cudaGetLastError();
    }
    return e;
  };
  auto mass_apply = [&](double* d) -> cudaError_t {
    icx::mass_apply_kernel<<<icx::grid_for(n), 256, 0, s>>>(dm.E, dm.nb, dm.neq, w->minv, w->singular, w->r, d);
    return cudaGetLastError();
  };
  XCK(residual(d_u));  // solve(): initial residual for the wave speeds
  int itime = 0;
  double time = 0.0, dt = 0.0, lam = 0.0;
  while (o->termination == 0 ? itime < o->ntime : time < o->tfinal) {
    dt = o->dt;
    if (o->timestep == 1) {
      unsigned long long bits = 0;
      XCK(cudaMemcpyAsync(&bits, w->lam, sizeof(bits), cudaMemcpyDeviceToHost, s));
      XCK(cudaStreamSynchronize(s));
      std::memcpy(&lam, &bits, sizeof(lam));
      // dt_from_cfl (burgers.hpp:104-108) / (2 Pn_max + 1) (explicit_utils.hpp:87-88)
      dt = (reflen * o->cfl) / (c->phys.mu / reflen + lam) / (2 * c->p + 1);
    }
    if (o->termination == 1) dt = std::min(dt, o->tfinal - time);
    if (o->scheme == 0) {
      XCK(residual(d_u));
      XCK(mass_apply(w->d1));
      icx::explicit_update_kernel<<<icx::grid_for(n), 256, 0, s>>>(n, d_u, dt, w->d1, 0.0, nullptr, 0.0, nullptr);
      XCK(cudaGetLastError());
    } else if (o->scheme == 1) {
      static const double alfa[3] = {0.0, 0.75, 1.0 / 3.0}, beta[3] = {1.0, 0.25, 2.0 / 3.0};
      XCK(cudaMemcpyAsync(w->uold, d_u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      for (int stg = 0; stg < 3; ++stg) {
        XCK(residual(d_u));
        XCK(mass_apply(w->d1));
        icx::tvd_stage_kernel<<<icx::grid_for(n), 256, 0, s>>>(n, d_u, w->uold, alfa[stg], beta[stg], beta[stg] * dt,
                                                               w->d1);
        XCK(cudaGetLastError());
      }
    } else {
      // every stage residual at the step's initial state, as the reference computes them
      double* ds[3] = {w->d1, w->d2, w->d3};
      for (int stg = 0; stg < 3; ++stg) {
        XCK(residual(d_u));
        XCK(mass_apply(ds[stg]));
      }
      icx::explicit_update_kernel<<<icx::grid_for(n), 256, 0, s>>>(n, d_u, 1.0 / 6.0 * dt, w->d1, 1.0 / 6.0 * dt, w->d2,
                                                                   2.0 / 3.0 * dt, w->d3);
      XCK(cudaGetLastError());
    }
    ++itime;
    time += dt;
  }
  XCK(cudaStreamSynchronize(s));
  if (rep) {
    rep->steps = itime;
    rep->time = time;
    rep->dt_last = dt;
    unsigned long long bits = 0;
    XCK(cudaMemcpy(&bits, w->lam, sizeof(bits), cudaMemcpyDeviceToHost));
    std::memcpy(&rep->lambda_max, &bits, sizeof(double));
    rep->singular_elements = ns;
  }
  return ICX_OK;
}

}  // extern "C"
