// Sets of independent problems of uneven mesh size and basis order, each
// solved by its own Newton iteration (PetscNewton::solve,
// src/solvers/include/iceicle/petsc_newton.hpp:205-329), all advanced
// together on one GPU.
//
// The parts are grouped by basis order; each group is one batch context
// (icx_batch_create): its kernels cover all parts of that order in one launch.
// What makes the solves independent is the reduction: every inner product,
// norm and stopping test is taken per part over that part's unknowns
// (segmented reductions over fixed-size chunks that never span two parts,
// summed in a fixed order, so results do not depend on the launch). Each part
// therefore has its own GMRES Krylov space, Hessenberg matrix, Givens
// rotations and convergence (right-preconditioned restarted GMRES, as
// icx_gmres_solve), its own line search (the reference's Wolfe or Corrigan
// search, replayed per part against a cache of evaluated step lengths: every
// round evaluates the residual of the whole set once, at each part's next
// requested step length) and its own step and stopping test. A part that has
// converged keeps its state; its rows still flow through the group kernels
// (their right-hand side is zero, so its update is zero).
//
// One Arnoldi step of the whole set (every group's preconditioner apply and
// Jacobian product, both Gram-Schmidt passes, the norm, the normalisation and
// the copy of the per-part Hessenberg column to the host) is one CUDA graph,
// captured on the step's second eager run and replayed afterwards.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "icx_internal.h"
#include "icx_linalg.h"

namespace {

constexpr long long kChunk = 4096;  // unknowns per reduction chunk (a chunk lies in one part)
constexpr int kThreads = 256;
constexpr int kPer = (int)(kChunk / kThreads);

// partial[c * ldp + j] = sum over chunk c of V_j . x   (V_j = V + j * ld)
__global__ void __launch_bounds__(kThreads) seg_dot_partial_kernel(const long long* __restrict__ cbeg,
                                                                   const long long* __restrict__ cend,
                                                                   const double* __restrict__ V, long long ld,
                                                                   int nvec, const double* __restrict__ x,
                                                                   double* __restrict__ partial, int ldp) {
  const int c = blockIdx.x;
  const long long b = cbeg[c], e = cend[c];
  double xv[kPer];
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const long long k = b + threadIdx.x + (long long)t * kThreads;
    xv[t] = k < e ? x[k] : 0.0;
  }
  __shared__ double red[kThreads / 32];
  for (int j = 0; j < nvec; ++j) {
    const double* v = V + (size_t)j * ld;
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const long long k = b + threadIdx.x + (long long)t * kThreads;
      if (k < e) s += v[k] * xv[t];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) a += red[w];
      partial[(size_t)c * ldp + j] = a;
    }
    __syncthreads();
  }
}

// out[p * ldo + j] = the partials of part p's chunks summed in ascending order
// (one warp per part, lanes over j)
__global__ void seg_dot_final_kernel(int n_parts, const int* __restrict__ pck, const double* __restrict__ partial,
                                     int ldp, int nvec, double* __restrict__ out, int ldo) {
  const int p = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (p >= n_parts) return;
  for (int j = threadIdx.x & 31; j < nvec; j += 32) {
    double s = 0.0;
    for (int c = pck[p]; c < pck[p + 1]; ++c) s += partial[(size_t)c * ldp + j];
    out[(size_t)p * ldo + j] = s;
  }
}

// w += sign * sum_j coef[part * ldc + j] V_j, chunk by chunk
__global__ void seg_maxpy_kernel(const long long* __restrict__ cbeg, const long long* __restrict__ cend,
                                 const int* __restrict__ cpart, const double* __restrict__ V, long long ld, int nvec,
                                 const double* __restrict__ coef, int ldc, double sign, double* __restrict__ w) {
  const int c = blockIdx.x;
  const double* h = coef + (size_t)cpart[c] * ldc;
  for (long long k = cbeg[c] + threadIdx.x; k < cend[c]; k += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < nvec; ++j) s += h[j] * V[(size_t)j * ld + k];
    w[k] += sign * s;
  }
}

// v = a[part] x   (a = 0 clears the part)
__global__ void seg_scale_kernel(const long long* __restrict__ cbeg, const long long* __restrict__ cend,
                                 const int* __restrict__ cpart, const double* __restrict__ a, int lda,
                                 const double* __restrict__ x, double* __restrict__ v) {
  const int c = blockIdx.x;
  const double s = a[(size_t)cpart[c] * lda];
  for (long long k = cbeg[c] + threadIdx.x; k < cend[c]; k += blockDim.x) v[k] = s * x[k];
}

// v /= sqrt(h2[part]) where h2 > 0 (as icx_gmres_solve: a = 1 / sqrt(h2), v = a v + 0 v)
__global__ void seg_normalize_kernel(const long long* __restrict__ cbeg, const long long* __restrict__ cend,
                                     const int* __restrict__ cpart, const double* __restrict__ h2, int ldh,
                                     double* __restrict__ v) {
  const int c = blockIdx.x;
  const double h = h2[(size_t)cpart[c] * ldh];
  if (!(h > 0.0)) return;
  const double a = 1.0 / sqrt(h);
  for (long long k = cbeg[c] + threadIdx.x; k < cend[c]; k += blockDim.x) v[k] = a * v[k] + 0.0 * v[k];
}

// z = x + a[part] y
__global__ void seg_xpay_kernel(const long long* __restrict__ cbeg, const long long* __restrict__ cend,
                                const int* __restrict__ cpart, const double* __restrict__ x,
                                const double* __restrict__ a, const double* __restrict__ y, double* __restrict__ z) {
  const int c = blockIdx.x;
  const double s = a[cpart[c]];
  for (long long k = cbeg[c] + threadIdx.x; k < cend[c]; k += blockDim.x) z[k] = x[k] + s * y[k];
}

// y = a[part] x + 1 y
__global__ void seg_axpy_kernel(const long long* __restrict__ cbeg, const long long* __restrict__ cend,
                                const int* __restrict__ cpart, const double* __restrict__ a,
                                const double* __restrict__ x, double* __restrict__ y) {
  const int c = blockIdx.x;
  const double s = a[cpart[c]];
  for (long long k = cbeg[c] + threadIdx.x; k < cend[c]; k += blockDim.x) y[k] = s * x[k] + 1.0 * y[k];
}

// the Hessenberg column of step j per part: both Gram-Schmidt passes summed
// (d1 null: one pass), then |v_j+1|^2 (the host takes the root)
__global__ void seg_hcol_kernel(int n_parts, int j, const double* __restrict__ d0, const double* __restrict__ d1,
                                const double* __restrict__ d2, int ld, double* __restrict__ hcol) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_parts * (j + 2)) return;
  const int p = t / (j + 2), i = t - p * (j + 2);
  hcol[(size_t)p * ld + i] = i <= j ? d0[(size_t)p * ld + i] + (d1 ? d1[(size_t)p * ld + i] : 0.0) : d2[(size_t)p * ld];
}

struct NeedEval {
  double alpha;
};

}  // namespace

struct icx_pset {
  int device = 0;
  int n_parts = 0;
  std::vector<icx_ctx*> groups;       // one batch context per basis order (owned)
  std::vector<long long> group_off;   // first unknown of each group
  std::vector<long long> group_n;
  std::vector<int> store_user;        // storage index -> caller's part index
  std::vector<long long> user_off;    // caller's part index -> first unknown
  long long N = 0;
  int n_chunks = 0;
  long long* d_cbeg = nullptr;
  long long* d_cend = nullptr;
  int* d_cpart = nullptr;             // chunk -> storage index
  int* d_pck = nullptr;               // storage index -> first chunk (n_parts + 1)
  // solver buffers (sized for restart m)
  int m = 0;
  double *V = nullptr, *w = nullptr, *z = nullptr, *r = nullptr, *res = nullptr, *du = nullptr, *ut = nullptr,
         *rt = nullptr;
  double* partial = nullptr;          // [n_chunks][m + 2]
  double* dots = nullptr;             // [3][n_parts][m + 2]
  double* coef = nullptr;             // [n_parts][m + 2]
  double* hcol = nullptr;             // [n_parts][m + 2]
  double* h_hcol = nullptr;           // pinned copy of hcol
  double* h_small = nullptr;          // pinned [n_parts][m + 2] staging
  cudaStream_t cap = nullptr;         // graph capture stream
  std::vector<cudaGraphExec_t> exec;  // Arnoldi step graphs (step j)
  std::vector<int> seen;
  unsigned long long key = 0;
  bool graphs_failed = false;
  std::string err;
};

namespace {

icx_status perr(icx_pset* S, icx_status st, const std::string& m) {
  if (S) S->err = m;
  return st;
}

#define PCK(expr)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess) return perr(S, ICX_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

void release_graphs(icx_pset* S) {
  for (cudaGraphExec_t& g : S->exec)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  std::fill(S->seen.begin(), S->seen.end(), 0);
  S->graphs_failed = false;
}

void free_buffers(icx_pset* S) {
  release_graphs(S);
  S->exec.clear();
  S->seen.clear();
  void* dev[] = {S->V, S->w, S->z, S->r, S->res, S->du, S->ut, S->rt, S->partial, S->dots, S->coef, S->hcol};
  for (void* p : dev)
    if (p) cudaFree(p);
  S->V = S->w = S->z = S->r = S->res = S->du = S->ut = S->rt = S->partial = S->dots = S->coef = S->hcol = nullptr;
  if (S->h_hcol) cudaFreeHost(S->h_hcol);
  if (S->h_small) cudaFreeHost(S->h_small);
  S->h_hcol = S->h_small = nullptr;
  S->m = 0;
}

icx_status ensure_buffers(icx_pset* S, int m) {
  if (S->m >= m) return ICX_OK;
  free_buffers(S);
  const size_t n = (size_t)S->N, ld = (size_t)m + 2, P = (size_t)S->n_parts;
  PCK(cudaMalloc((void**)&S->V, sizeof(double) * (m + 1) * n));
  double** vecs[] = {&S->w, &S->z, &S->r, &S->res, &S->du, &S->ut, &S->rt};
  for (double** p : vecs) PCK(cudaMalloc((void**)p, sizeof(double) * n));
  PCK(cudaMalloc((void**)&S->partial, sizeof(double) * (size_t)S->n_chunks * ld));
  PCK(cudaMalloc((void**)&S->dots, sizeof(double) * 3 * P * ld));
  PCK(cudaMalloc((void**)&S->coef, sizeof(double) * P * ld));
  PCK(cudaMalloc((void**)&S->hcol, sizeof(double) * P * ld));
  PCK(cudaMallocHost((void**)&S->h_hcol, sizeof(double) * P * ld));
  PCK(cudaMallocHost((void**)&S->h_small, sizeof(double) * P * ld));
  S->exec.assign(m, nullptr);
  S->seen.assign(m, 0);
  S->m = m;
  return ICX_OK;
}

// out[p * ldo + j] = (V_j . x) over part p, j < nvec
cudaError_t seg_dots(icx_pset* S, const double* V, long long ld, int nvec, const double* x, double* out, int ldo,
                     cudaStream_t s) {
  const int ldp = S->m + 2;
  seg_dot_partial_kernel<<<S->n_chunks, kThreads, 0, s>>>(S->d_cbeg, S->d_cend, V, ld, nvec, x, S->partial, ldp);
  seg_dot_final_kernel<<<(S->n_parts + 7) / 8, 256, 0, s>>>(S->n_parts, S->d_pck, S->partial, ldp, nvec, out, ldo);
  return cudaGetLastError();
}

// per-part 2-norms of x into host[p] (synchronises)
icx_status seg_norms(icx_pset* S, const double* x, std::vector<double>& host, cudaStream_t s) {
  const int ld = S->m + 2;
  PCK(seg_dots(S, x, 0, 1, x, S->dots, ld, s));
  PCK(cudaMemcpyAsync(S->h_small, S->dots, sizeof(double) * S->n_parts * ld, cudaMemcpyDeviceToHost, s));
  PCK(cudaStreamSynchronize(s));
  host.resize(S->n_parts);
  for (int p = 0; p < S->n_parts; ++p) host[p] = std::sqrt(S->h_small[(size_t)p * ld]);
  return ICX_OK;
}

// a per-part scalar array on the device (coef[p * lda]) from host values
cudaError_t put_per_part(icx_pset* S, const std::vector<double>& v, double* dst, int lda, cudaStream_t s) {
  for (int p = 0; p < S->n_parts; ++p) S->h_small[(size_t)p * lda] = v[p];
  return cudaMemcpyAsync(dst, S->h_small, sizeof(double) * S->n_parts * lda, cudaMemcpyHostToDevice, s);
}

cudaError_t all_groups(icx_pset* S, const std::function<cudaError_t(icx_ctx*, long long)>& f) {
  for (size_t g = 0; g < S->groups.size(); ++g) {
    cudaError_t e = f(S->groups[g], S->group_off[g]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

struct Kry {
  double bnorm = 0.0, tol = 0.0, beta = 0.0, relres = 0.0, resid = 0.0;
  int total = 0, jdim = 0;
  bool done = true, in_cycle = false;
  std::vector<double> H, cs, sn, g, y;
};

// x = J^-1 b per part (parts with want[p] = 0 keep x = 0): restarted
// right-preconditioned GMRES(m) of each part, all parts in the same launches
icx_status pset_gmres(icx_pset* S, int pc, bool mixed, int m, int maxit, double rtol, const double* b, double* x,
                      const std::vector<char>& want, std::vector<int>& iters, std::vector<double>& relres,
                      icx_pset_stats& st, cudaStream_t s, int passes = 2) {
  const int P = S->n_parts, ld = m + 2;
  const long long N = S->N;
  PCK(cudaMemsetAsync(x, 0, sizeof(double) * N, s));
  std::vector<double> bn;
  icx_status rs = seg_norms(S, b, bn, s);
  if (rs != ICX_OK) return rs;
  std::vector<Kry> K(P);
  for (int p = 0; p < P; ++p) {
    K[p].bnorm = bn[p];
    K[p].done = !want[p] || bn[p] == 0.0;
    if (want[p] && !std::isfinite(bn[p])) return perr(S, ICX_ERR_NONFINITE, "non-finite right-hand side");
    K[p].tol = rtol * bn[p];
    K[p].beta = bn[p];
    K[p].H.assign((size_t)(m + 1) * m, 0.0);
    K[p].cs.assign(m, 0.0);
    K[p].sn.assign(m, 0.0);
    K[p].g.assign(m + 1, 0.0);
    K[p].y.assign(m, 0.0);
  }
  PCK(cudaMemcpyAsync(S->r, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  // graphs of the Arnoldi steps, valid while the key holds
  bool graphable = true;
  unsigned long long key = 1469598103934665603ull;
  for (icx_ctx* g : S->groups) {
    graphable = graphable && icx::solver_graphable(g, pc, mixed);
    key = (key ^ icx::solver_graph_key(g, pc, mixed)) * 1099511628211ull;
  }
  key = (key ^ (unsigned long long)m) * 1099511628211ull;
  key = (key ^ (unsigned long long)passes) * 1099511628211ull;
  if (key != S->key) {
    release_graphs(S);
    S->key = key;
  }
  if (graphable && !S->cap && cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking) != cudaSuccess)
    graphable = false;
  std::vector<double> a(P);
  while (true) {
    bool any = false;
    for (int p = 0; p < P; ++p) {
      Kry& k = K[p];
      k.in_cycle = !k.done;
      k.jdim = 0;
      any = any || k.in_cycle;
      a[p] = k.in_cycle ? 1.0 / k.beta : 0.0;
      std::fill(k.g.begin(), k.g.end(), 0.0);
      k.g[0] = k.beta;
    }
    if (!any) break;
    PCK(put_per_part(S, a, S->coef, ld, s));
    seg_scale_kernel<<<S->n_chunks, kThreads, 0, s>>>(S->d_cbeg, S->d_cend, S->d_cpart, S->coef, ld, S->r, S->V);
    PCK(cudaGetLastError());
    int j = 0;
    for (; j < m; ++j) {
      bool live = false;
      for (int p = 0; p < P; ++p) live = live || K[p].in_cycle;
      if (!live) break;
      double* vj = S->V + (size_t)j * N;
      double* vj1 = S->V + (size_t)(j + 1) * N;
      auto step = [&](cudaStream_t q) -> cudaError_t {
        cudaError_t e = all_groups(S, [&](icx_ctx* g, long long off) -> cudaError_t {
          cudaError_t ee = pc ? icx::solver_apply_pc(g, pc, mixed, vj + off, S->z + off, q) : cudaSuccess;
          if (ee == cudaSuccess) ee = icx::solver_operator(g, mixed, (pc ? S->z : vj) + off, vj1 + off, q);
          return ee;
        });
        for (int pass = 0; pass < passes && e == cudaSuccess; ++pass) {
          double* slot = S->dots + (size_t)pass * P * ld;
          e = seg_dots(S, S->V, N, j + 1, vj1, slot, ld, q);
          if (e == cudaSuccess) {
            seg_maxpy_kernel<<<S->n_chunks, kThreads, 0, q>>>(S->d_cbeg, S->d_cend, S->d_cpart, S->V, N, j + 1, slot, ld,
                                                             -1.0, vj1);
            e = cudaGetLastError();
          }
        }
        double* nrm = S->dots + (size_t)2 * P * ld;
        if (e == cudaSuccess) e = seg_dots(S, vj1, 0, 1, vj1, nrm, ld, q);
        if (e == cudaSuccess) {
          seg_hcol_kernel<<<(P * (j + 2) + 255) / 256, 256, 0, q>>>(
              P, j, S->dots, passes == 2 ? S->dots + (size_t)P * ld : nullptr, nrm, ld, S->hcol);
          seg_normalize_kernel<<<S->n_chunks, kThreads, 0, q>>>(S->d_cbeg, S->d_cend, S->d_cpart, nrm, ld, vj1);
          e = cudaGetLastError();
        }
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(S->h_hcol, S->hcol, sizeof(double) * P * ld, cudaMemcpyDeviceToHost, q);
        return e;
      };
      cudaGraphExec_t gx = nullptr;
      if (graphable && !S->graphs_failed) {
        if (S->exec[j]) {
          gx = S->exec[j];
        } else if (S->seen[j]++ >= 1) {
          // capture on the step's second eager run: the first has done every
          // one-time setup of the kernels it launches
          cudaGraph_t graph = nullptr;
          cudaError_t e = cudaStreamBeginCapture(S->cap, cudaStreamCaptureModeThreadLocal);
          if (e == cudaSuccess) {
            cudaError_t es = step(S->cap);
            e = cudaStreamEndCapture(S->cap, &graph);
            if (es != cudaSuccess) e = es;
          }
          if (e == cudaSuccess) e = cudaGraphInstantiate(&S->exec[j], graph, 0);
          if (graph) cudaGraphDestroy(graph);
          if (e != cudaSuccess) {
            (void)cudaGetLastError();
            S->exec[j] = nullptr;
            S->graphs_failed = true;
          }
          gx = S->exec[j];
        }
      }
      if (gx) {
        PCK(cudaGraphLaunch(gx, s));
        ++st.graph_launches;
      } else {
        PCK(step(s));
      }
      PCK(cudaStreamSynchronize(s));
      ++st.arnoldi_steps;
      for (int p = 0; p < P; ++p) {
        Kry& k = K[p];
        if (!k.in_cycle) continue;
        const double* hc = S->h_hcol + (size_t)p * ld;
        std::vector<double> col(hc, hc + j + 1);
        const double hn = std::sqrt(hc[j + 1]);
        if (!std::isfinite(hn)) return perr(S, ICX_ERR_NONFINITE, "non-finite Krylov vector");
        col.push_back(hn);
        for (int i = 0; i < j; ++i) {
          const double t = k.cs[i] * col[i] + k.sn[i] * col[i + 1];
          col[i + 1] = -k.sn[i] * col[i] + k.cs[i] * col[i + 1];
          col[i] = t;
        }
        const double den = std::hypot(col[j], col[j + 1]);
        k.cs[j] = den == 0.0 ? 1.0 : col[j] / den;
        k.sn[j] = den == 0.0 ? 0.0 : col[j + 1] / den;
        col[j] = den;
        k.g[j + 1] = -k.sn[j] * k.g[j];
        k.g[j] = k.cs[j] * k.g[j];
        for (int i = 0; i <= j; ++i) k.H[(size_t)i * m + j] = col[i];
        ++k.total;
        k.jdim = j + 1;
        k.resid = std::fabs(k.g[j + 1]);
        if (k.resid <= k.tol || hn == 0.0 || k.total >= maxit) k.in_cycle = false;
      }
    }
    // x += M^-1 (V y) per part
    int jmax = 0;
    for (int p = 0; p < P; ++p) {
      Kry& k = K[p];
      std::fill(k.y.begin(), k.y.end(), 0.0);
      for (int i = k.jdim - 1; i >= 0; --i) {
        double sacc = k.g[i];
        for (int q = i + 1; q < k.jdim; ++q) sacc -= k.H[(size_t)i * m + q] * k.y[q];
        k.y[i] = sacc / k.H[(size_t)i * m + i];
      }
      jmax = std::max(jmax, k.jdim);
      for (int i = 0; i < m + 2; ++i) S->h_small[(size_t)p * ld + i] = i < m ? k.y[i] : 0.0;
    }
    PCK(cudaMemcpyAsync(S->coef, S->h_small, sizeof(double) * P * ld, cudaMemcpyHostToDevice, s));
    PCK(cudaMemsetAsync(S->w, 0, sizeof(double) * N, s));
    if (jmax > 0) {
      seg_maxpy_kernel<<<S->n_chunks, kThreads, 0, s>>>(S->d_cbeg, S->d_cend, S->d_cpart, S->V, N, jmax, S->coef, ld,
                                                       1.0, S->w);
      PCK(cudaGetLastError());
    }
    if (pc) {
      PCK(all_groups(S, [&](icx_ctx* g, long long off) {
        return icx::solver_apply_pc(g, pc, mixed, S->w + off, S->z + off, s);
      }));
      PCK(icx::la_axpby(N, 1.0, S->z, 1.0, x, s));
    } else {
      PCK(icx::la_axpby(N, 1.0, S->w, 1.0, x, s));
    }
    PCK(all_groups(S, [&](icx_ctx* g, long long off) { return icx::solver_operator(g, mixed, x + off, S->w + off, s); }));
    PCK(icx::la_xpay(N, b, -1.0, S->w, S->r, s));
    std::vector<double> beta;
    rs = seg_norms(S, S->r, beta, s);
    if (rs != ICX_OK) return rs;
    for (int p = 0; p < P; ++p) {
      Kry& k = K[p];
      if (k.done || k.jdim == 0) continue;
      k.beta = beta[p];
      k.relres = k.beta / k.bnorm;
      if (k.beta <= k.tol || k.total >= maxit || k.resid <= k.tol) k.done = true;
    }
  }
  iters.assign(P, 0);
  relres.assign(P, 0.0);
  for (int p = 0; p < P; ++p) {
    iters[p] = K[p].total;
    relres[p] = K[p].relres;
  }
  // an abandoned data-flow apply leaves its error flag set
  for (icx_ctx* g : S->groups) {
    int fl = 0;
    if (icx::solver_take_pc_err(g, &fl) != ICX_OK) return perr(S, ICX_ERR_CUDA, "reading the apply's error flag");
    if (fl) return perr(S, ICX_ERR_CUDA, fl == 2 ? "block-ILU apply: block index out of range"
                                                 : "block-ILU apply: a dependency wait timed out");
  }
  return ICX_OK;
}

}  // namespace

extern "C" {

icx_status icx_pset_create(icx_pset** out, int device, int n_parts, icx_ctx* const* parts) {
  if (!out || n_parts < 1 || !parts) return ICX_ERR_INVALID;
  *out = nullptr;
  for (int k = 0; k < n_parts; ++k) {
    if (!parts[k] || !parts[k]->ready || !parts[k]->parts.empty()) return ICX_ERR_INVALID;
    if (parts[k]->phys.pde != parts[0]->phys.pde) return ICX_ERR_INVALID;
  }
  icx_pset* S = new icx_pset();
  S->device = device;
  S->n_parts = n_parts;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete S;
    return ICX_ERR_CUDA;
  }
  std::map<int, std::vector<int>> by_p;
  for (int k = 0; k < n_parts; ++k) by_p[parts[k]->p].push_back(k);
  S->user_off.assign(n_parts + 1, 0);
  std::vector<long long> len;
  for (auto& kv : by_p) {
    std::vector<icx_ctx*> members;
    for (int k : kv.second) members.push_back(parts[k]);
    icx_ctx* g = nullptr;
    icx_status st = icx_batch_create(&g, device, (int)members.size(), members.data());
    if (st != ICX_OK) {
      icx_pset_destroy(S);
      return st;
    }
    S->groups.push_back(g);
    S->group_off.push_back(S->N);
    long long gn = 0;
    for (int k : kv.second) {
      const icx_ctx* q = parts[k];
      const long long nk = (long long)q->dm.E * q->dm.nb * q->dm.neq;
      S->user_off[k] = S->N + gn;
      S->store_user.push_back(k);
      len.push_back(nk);
      gn += nk;
    }
    S->group_n.push_back(gn);
    S->N += gn;
  }
  S->user_off[n_parts] = S->N;
  // reduction chunks in storage order
  std::vector<long long> cb, ce;
  std::vector<int> cp, pck(n_parts + 1, 0);
  long long off = 0;
  for (int sp = 0; sp < n_parts; ++sp) {
    pck[sp] = (int)cb.size();
    for (long long b = 0; b < len[sp]; b += kChunk) {
      cb.push_back(off + b);
      ce.push_back(off + std::min(len[sp], b + kChunk));
      cp.push_back(sp);
    }
    off += len[sp];
  }
  pck[n_parts] = (int)cb.size();
  S->n_chunks = (int)cb.size();
  bool ok = cudaMalloc((void**)&S->d_cbeg, sizeof(long long) * cb.size()) == cudaSuccess &&
            cudaMalloc((void**)&S->d_cend, sizeof(long long) * ce.size()) == cudaSuccess &&
            cudaMalloc((void**)&S->d_cpart, sizeof(int) * cp.size()) == cudaSuccess &&
            cudaMalloc((void**)&S->d_pck, sizeof(int) * pck.size()) == cudaSuccess &&
            cudaMemcpy(S->d_cbeg, cb.data(), sizeof(long long) * cb.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(S->d_cend, ce.data(), sizeof(long long) * ce.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(S->d_cpart, cp.data(), sizeof(int) * cp.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(S->d_pck, pck.data(), sizeof(int) * pck.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    icx_pset_destroy(S);
    return ICX_ERR_CUDA;
  }
  *out = S;
  return ICX_OK;
}

void icx_pset_destroy(icx_pset* S) {
  if (!S) return;
  cudaSetDevice(S->device);
  free_buffers(S);
  if (S->cap) cudaStreamDestroy(S->cap);
  void* dev[] = {S->d_cbeg, S->d_cend, S->d_cpart, S->d_pck};
  for (void* p : dev)
    if (p) cudaFree(p);
  for (icx_ctx* g : S->groups) icx_destroy(g);
  delete S;
}

icx_status icx_pset_offsets(const icx_pset* S, long long* offsets) {
  if (!S || !offsets) return ICX_ERR_INVALID;
  std::copy(S->user_off.begin(), S->user_off.end(), offsets);
  return ICX_OK;
}

const char* icx_pset_last_error(const icx_pset* S) { return S ? S->err.c_str() : "null set"; }

icx_status icx_pset_residual(icx_pset* S, const double* d_u, double* d_res) {
  if (!S || !d_u || !d_res) return ICX_ERR_INVALID;
  cudaSetDevice(S->device);
  cudaStream_t s = 0;
  PCK(all_groups(S, [&](icx_ctx* g, long long off) {
    return icx::launch_residual(g->dm, g->phys, d_u + off, d_res + off, s);
  }));
  PCK(cudaStreamSynchronize(s));
  return ICX_OK;
}

icx_status icx_pset_newton_solve(icx_pset* S, double* d_u, const icx_newton_options* opt,
                                 icx_newton_report* reports, icx_pset_stats* stats) {
  if (!S || !d_u || !opt) return ICX_ERR_INVALID;
  if (opt->gmres_restart < 1 || opt->gmres_restart > 60) return perr(S, ICX_ERR_INVALID, "restart in 1..60");
  if (opt->precision < 0 || opt->precision > 2) return perr(S, ICX_ERR_INVALID, "precision must be 0, 1 or 2");
  if (!(opt->preconditioner >= 0 && opt->preconditioner <= 2) && opt->preconditioner != 4)
    return perr(S, ICX_ERR_INVALID, "preconditioner 0, 1, 2 or 4 on a set");
  if (opt->preconditioner == 4 && (opt->pc_sweeps < 0 || opt->pc_sweeps > 16))
    return perr(S, ICX_ERR_INVALID, "pc_sweeps in 0..16");
  cudaSetDevice(S->device);
  cudaStream_t s = 0;
  const int P = S->n_parts, m = opt->gmres_restart, pc = opt->preconditioner;
  const bool mixed = opt->precision >= 1;
  icx_status st = ensure_buffers(S, m);
  if (st != ICX_OK) return st;
  for (icx_ctx* g : S->groups) {
    st = icx::solver_group_ready(g, opt->precision, opt->pc_sweeps, opt->ilu_tile, opt->cuda_graphs != 0);
    if (st != ICX_OK) return perr(S, st, std::string("group solver buffers: ") + g->err);
  }
  icx_pset_stats local_stats{};
  icx_pset_stats& stt = stats ? *stats : local_stats;
  std::memset(&stt, 0, sizeof(stt));
  stt.orders = (int)S->groups.size();
  std::vector<icx_newton_report> R(P);
  for (auto& r : R) std::memset(&r, 0, sizeof(r));
  auto linearise = [&]() -> cudaError_t {
    return all_groups(S, [&](icx_ctx* g, long long off) {
      return icx::solver_linearise(g, d_u + off, S->res + off, opt->precision, s);
    });
  };
  PCK(linearise());
  std::vector<double> rk;
  st = seg_norms(S, S->res, rk, s);
  if (st != ICX_OK) return st;
  std::vector<char> active(P, 0), failed(P, 0);
  std::vector<double> tau(P);
  for (int p = 0; p < P; ++p) {
    R[p].r0 = rk[p];
    R[p].residual_history[0] = rk[p];
    R[p].r_final = rk[p];
    tau[p] = opt->tau_abs + opt->tau_rel * rk[p];
    if (!std::isfinite(rk[p])) failed[p] = 1;
    active[p] = !failed[p] && !(rk[p] <= tau[p]);
  }
  std::vector<int> its;
  std::vector<double> rel, alpha(P), a_dev(P);
  for (int k = 0; k < opt->kmax; ++k) {
    bool any = false;
    for (int p = 0; p < P; ++p) any = any || active[p];
    if (!any) break;
    ++stt.newton_rounds;
    PCK(all_groups(S, [&](icx_ctx* g, long long) { return icx::solver_build_pc(g, pc, mixed, s); }));
    for (icx_ctx* g : S->groups) {
      int fl = 0;
      PCK(cudaMemcpyAsync(&fl, icx::solver_flag(g), sizeof(int), cudaMemcpyDeviceToHost, s));
      PCK(cudaStreamSynchronize(s));
      if (fl == 2) return perr(S, ICX_ERR_CUDA, "block-ILU factorization: block index out of range");
    }
    st = pset_gmres(S, pc, mixed, m, opt->gmres_max_it, opt->gmres_rtol, S->res, S->du, active, its, rel, stt, s,
                    opt->gmres_cgs_refine ? 2 : 1);
    if (st != ICX_OK) return st;
    for (int p = 0; p < P; ++p) {
      if (!active[p]) continue;
      R[p].linear_iterations_total += its[p];
      if (k < 64) R[p].linear_iterations[k] = its[p];
    }
    // each part's line search, replayed against its cache of evaluated step
    // lengths; one residual evaluation of the whole set per round
    std::fill(alpha.begin(), alpha.end(), 0.0);
    if (opt->linesearch != 0) {
      std::vector<std::map<double, double>> cache(P);
      std::vector<char> ls_done(P, 0);
      for (int p = 0; p < P; ++p)
        if (active[p]) cache[p][0.0] = R[p].r_final;
      for (int round = 0;; ++round) {
        bool need = false;
        std::vector<double> want_alpha(P, 0.0);
        std::vector<char> asked(P, 0);
        for (int p = 0; p < P; ++p) {
          if (!active[p] || ls_done[p]) continue;
          std::map<double, double>& C = cache[p];
          std::function<double(double)> f = [&C](double a) -> double {
            auto it = C.find(a);
            if (it == C.end()) throw NeedEval{a};
            return it->second;
          };
          try {
            alpha[p] = icx::solver_line_search(opt->linesearch, f, *opt);
            ls_done[p] = 1;
          } catch (const NeedEval& ne) {
            want_alpha[p] = ne.alpha;
            asked[p] = 1;
            need = true;
          }
        }
        if (!need) break;
        for (int p = 0; p < P; ++p) a_dev[p] = -want_alpha[p];
        PCK(put_per_part(S, a_dev, S->coef, 1, s));
        seg_xpay_kernel<<<S->n_chunks, kThreads, 0, s>>>(S->d_cbeg, S->d_cend, S->d_cpart, d_u, S->coef, S->du,
                                                        S->ut);
        PCK(cudaGetLastError());
        PCK(all_groups(S, [&](icx_ctx* g, long long off) {
          return icx::launch_residual(g->dm, g->phys, S->ut + off, S->rt + off, s);
        }));
        std::vector<double> phi;
        st = seg_norms(S, S->rt, phi, s);
        if (st != ICX_OK) return st;
        ++stt.line_search_rounds;
        for (int p = 0; p < P; ++p)
          if (asked[p]) cache[p][want_alpha[p]] = std::isfinite(phi[p]) ? phi[p] : 1e9;
      }
    } else {
      for (int p = 0; p < P; ++p) alpha[p] = active[p] ? 1.0 : 0.0;
    }
    for (int p = 0; p < P; ++p) a_dev[p] = active[p] ? -alpha[p] : 0.0;
    PCK(put_per_part(S, a_dev, S->coef, 1, s));
    seg_axpy_kernel<<<S->n_chunks, kThreads, 0, s>>>(S->d_cbeg, S->d_cend, S->d_cpart, S->coef, S->du, d_u);
    PCK(cudaGetLastError());
    PCK(linearise());
    st = seg_norms(S, S->res, rk, s);
    if (st != ICX_OK) return st;
    for (int p = 0; p < P; ++p) {
      if (!active[p]) continue;
      const int kk = R[p].iterations;
      if (kk + 1 < 64) {
        R[p].residual_history[kk + 1] = rk[p];
        R[p].alpha_history[kk] = alpha[p];
      }
      R[p].iterations = kk + 1;
      R[p].r_final = rk[p];
      if (opt->verbosity > 0)
        std::printf("part %d newton %d: |r| = %.6e alpha = %.4f gmres its = %d\n", S->store_user[p], kk, rk[p],
                    alpha[p], its[p]);
      if (!std::isfinite(rk[p])) {
        failed[p] = 1;
        active[p] = 0;
      } else if (rk[p] <= tau[p]) {
        active[p] = 0;
      }
    }
  }
  PCK(cudaStreamSynchronize(s));
  bool all_conv = true;
  for (int p = 0; p < P; ++p) {
    R[p].converged = !failed[p] && R[p].r_final <= tau[p];
    all_conv = all_conv && R[p].converged;
    if (reports) reports[S->store_user[p]] = R[p];
  }
  if (!all_conv) S->err = "a part did not converge (see its report)";
  return all_conv ? ICX_OK : ICX_ERR_NOT_CONVERGED;
}

}  // extern "C"
