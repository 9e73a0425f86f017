// Device linear algebra for the Newton solver: block-diagonal inversion
// (block-Jacobi preconditioner), block-ILU(0) on the element block pattern,
// deterministic reductions and the multi-vector kernels of GMRES.
#include <cfloat>
#include <cmath>
#include <vector>

#include "icx_internal.h"
#include "icx_linalg.h"

namespace icx {

// ----------------------------------------------------- block inversion
// In-place Gauss-Jordan inversion with partial pivoting of one bs x bs block
// per CTA, in shared memory. A singular pivot leaves the block as identity and
// raises *flag (the preconditioner degrades to no-op on that block).
__global__ void block_invert_kernel(int nblk, int bs, const double* __restrict__ src, const int* __restrict__ blk_index,
                                    double* __restrict__ dst, int* flag) {
  extern __shared__ double a[];
  int* perm = reinterpret_cast<int*>(a + bs * bs);
  __shared__ int piv_row;
  __shared__ double piv_val;
  __shared__ int singular;
  int b = blockIdx.x;
  if (b >= nblk) return;
  const double* A = src + (size_t)blk_index[b] * bs * bs;
  for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) a[t] = A[t];
  if (threadIdx.x == 0) singular = 0;
  __syncthreads();
  for (int k = 0; k < bs; ++k) {
    if (threadIdx.x == 0) {
      int p = k;
      double best = fabs(a[k * bs + k]);
      for (int i = k + 1; i < bs; ++i) {
        double v = fabs(a[i * bs + k]);
        if (v > best) { best = v; p = i; }
      }
      piv_row = p;
      perm[k] = p;
      if (best == 0.0) singular = 1;
      piv_val = a[p * bs + k];
    }
    __syncthreads();
    if (singular) break;
    int p = piv_row;
    if (p != k)
      for (int j = threadIdx.x; j < bs; j += blockDim.x) {
        double t = a[k * bs + j];
        a[k * bs + j] = a[p * bs + j];
        a[p * bs + j] = t;
      }
    __syncthreads();
    double pv = piv_val;
    for (int j = threadIdx.x; j < bs; j += blockDim.x) a[k * bs + j] = (j == k ? 1.0 : a[k * bs + j]) / pv;
    __syncthreads();
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) {
      int i = t / bs, j = t - i * bs;
      if (i == k) continue;
      double fct = a[i * bs + k];
      if (j == k) continue;
      a[t] -= fct * a[k * bs + j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < bs; i += blockDim.x)
      if (i != k) a[i * bs + k] = -a[i * bs + k] * a[k * bs + k];
    __syncthreads();
  }
  if (singular) {
    if (threadIdx.x == 0) atomicExch(flag, 1);
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) a[t] = (t / bs == t % bs) ? 1.0 : 0.0;
    __syncthreads();
  } else {
    // undo the row interchanges as column interchanges, in reverse order
    for (int k = bs - 1; k >= 0; --k) {
      int p = perm[k];
      if (p != k)
        for (int i = threadIdx.x; i < bs; i += blockDim.x) {
          double t = a[i * bs + k];
          a[i * bs + k] = a[i * bs + p];
          a[i * bs + p] = t;
        }
      __syncthreads();
    }
  }
  double* D = dst + (size_t)b * bs * bs;
  for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) D[t] = a[t];
}

// y_e = D_e x_e for block-diagonal D (one warp per block row)
template <int BS>
__global__ void block_diag_apply_kernel(int E, const double* __restrict__ D, const double* __restrict__ x,
                                        double* __restrict__ y) {
  int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (row >= E) return;
  const double* xv = x + (size_t)row * BS;
  for (int r = lane; r < BS; r += 32) {
    const double* A = D + (size_t)row * BS * BS + (size_t)r * BS;
    double acc = 0.0;
#pragma unroll 4
    for (int c = 0; c < BS; ++c) acc += A[c] * xv[c];
    y[(size_t)row * BS + r] = acc;
  }
}

// ------------------------------------------------------------ block-ILU(0)
// Block ILU(0) on the element block pattern in natural (element) order, IKJ
// form: for each row e, for each lower block (e, k) in ascending k,
//   A_ek <- A_ek inv(A_kk);  A_ej -= A_ek A_kj  for every (k, j), j > k, with (e, j) in the pattern;
// then inv(A_ee) is stored for the next rows and the backward solve. On the
// structured element grid row (i, j) depends only on (i-1, j) and (i, j-1),
// so the rows of one anti-diagonal i + j = level are independent: one launch
// per level, one CTA per row.

// Gauss-Jordan inversion of the bs x bs block in shared memory `a` (in place)
__device__ void gj_invert_shared(double* a, int* perm, int bs, int* s_flag, double* s_pv, int* s_pr) {
  for (int k = 0; k < bs; ++k) {
    if (threadIdx.x == 0) {
      int p = k;
      double best = fabs(a[k * bs + k]);
      for (int i = k + 1; i < bs; ++i) {
        double v = fabs(a[i * bs + k]);
        if (v > best) { best = v; p = i; }
      }
      *s_pr = p;
      perm[k] = p;
      if (best == 0.0) *s_flag = 1;
      *s_pv = a[p * bs + k];
    }
    __syncthreads();
    if (*s_flag) return;
    int p = *s_pr;
    if (p != k)
      for (int j = threadIdx.x; j < bs; j += blockDim.x) {
        double t = a[k * bs + j];
        a[k * bs + j] = a[p * bs + j];
        a[p * bs + j] = t;
      }
    __syncthreads();
    double pv = *s_pv;
    for (int j = threadIdx.x; j < bs; j += blockDim.x) a[k * bs + j] = (j == k ? 1.0 : a[k * bs + j]) / pv;
    __syncthreads();
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) {
      int i = t / bs, j = t - i * bs;
      if (i == k || j == k) continue;
      a[t] -= a[i * bs + k] * a[k * bs + j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < bs; i += blockDim.x)
      if (i != k) a[i * bs + k] = -a[i * bs + k] * a[k * bs + k];
    __syncthreads();
  }
  for (int k = bs - 1; k >= 0; --k) {
    int p = perm[k];
    if (p != k)
      for (int i = threadIdx.x; i < bs; i += blockDim.x) {
        double t = a[i * bs + k];
        a[i * bs + k] = a[i * bs + p];
        a[i * bs + p] = t;
      }
    __syncthreads();
  }
}

__device__ inline int find_block(const int* rowptr, const int* colidx, int r, int c) {
  for (int k = rowptr[r]; k < rowptr[r + 1]; ++k)
    if (colidx[k] == c) return k;
  return -1;
}

__global__ void ilu_level_kernel(int nx, int ny, int level, int bs, const int* __restrict__ rowptr,
                                 const int* __restrict__ colidx, double* __restrict__ LU, double* __restrict__ Uinv,
                                 int* flag) {
  extern __shared__ double sh[];
  double* Lek = sh;                                  // bs x bs
  double* Ainv = sh + bs * bs;                       // bs x bs
  int* perm = reinterpret_cast<int*>(sh + 2 * bs * bs);
  __shared__ int s_flag, s_pr;
  __shared__ double s_pv;
  int i0 = max(0, level - (ny - 1));
  int i = i0 + blockIdx.x, j = level - i;
  if (i >= nx || j < 0) return;
  int e = i + nx * j;
  if (threadIdx.x == 0) s_flag = 0;
  for (int kl = rowptr[e]; kl < rowptr[e + 1]; ++kl) {
    int k = colidx[kl];
    if (k >= e) break;  // columns ascend: the lower blocks come first
    double* Aek = LU + (size_t)kl * bs * bs;
    const double* Ui = Uinv + (size_t)k * bs * bs;
    __syncthreads();
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) {
      int r = t / bs, c = t - r * bs;
      double s = 0.0;
      for (int m = 0; m < bs; ++m) s += Aek[r * bs + m] * Ui[m * bs + c];
      Lek[t] = s;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) Aek[t] = Lek[t];
    for (int kj = rowptr[k]; kj < rowptr[k + 1]; ++kj) {
      int jc = colidx[kj];
      if (jc <= k) continue;
      int ej = find_block(rowptr, colidx, e, jc);
      if (ej < 0) continue;  // outside the pattern: dropped (level 0 fill)
      const double* Akj = LU + (size_t)kj * bs * bs;
      double* Aej = LU + (size_t)ej * bs * bs;
      __syncthreads();
      for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) {
        int r = t / bs, c = t - r * bs;
        double s = 0.0;
        for (int m = 0; m < bs; ++m) s += Lek[r * bs + m] * Akj[m * bs + c];
        Aej[t] -= s;
      }
    }
  }
  __syncthreads();
  int kd = find_block(rowptr, colidx, e, e);
  const double* Aee = LU + (size_t)kd * bs * bs;
  for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) Ainv[t] = Aee[t];
  __syncthreads();
  gj_invert_shared(Ainv, perm, bs, &s_flag, &s_pv, &s_pr);
  __syncthreads();
  double* D = Uinv + (size_t)e * bs * bs;
  if (s_flag) {
    if (threadIdx.x == 0) atomicExch(flag, 1);
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) D[t] = (t / bs == t % bs) ? 1.0 : 0.0;
  } else {
    for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) D[t] = Ainv[t];
  }
}

// one level of the triangular solves, one warp per block row:
//   forward  (ascending levels):  y_e = x_e - sum_{k<e} L_ek y_k
//   backward (descending levels): y_e = inv(U_ee) (y_e - sum_{k>e} U_ek y_k)
template <int BS>
__global__ void ilu_solve_level_kernel(int nx, int ny, int level, int forward, const int* __restrict__ rowptr,
                                       const int* __restrict__ colidx, const double* __restrict__ LU,
                                       const double* __restrict__ Uinv, const double* __restrict__ x,
                                       double* __restrict__ y) {
  __shared__ double tmp[4][BS];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int i0 = max(0, level - (ny - 1));
  int i = i0 + blockIdx.x * 4 + warp;
  int j = level - i;
  bool active = i < nx && j >= 0;
  int e = active ? i + nx * j : 0;
  if (active) {
    for (int r = lane; r < BS; r += 32) {
      double acc = forward ? x[(size_t)e * BS + r] : y[(size_t)e * BS + r];
      for (int k = rowptr[e]; k < rowptr[e + 1]; ++k) {
        int c = colidx[k];
        if (forward ? (c < e) : (c > e)) {
          const double* A = LU + (size_t)k * BS * BS + (size_t)r * BS;
          const double* v = y + (size_t)c * BS;
          for (int m = 0; m < BS; ++m) acc -= A[m] * v[m];
        }
      }
      tmp[warp][r] = acc;
    }
  }
  __syncwarp();
  if (active) {
    if (forward) {
      for (int r = lane; r < BS; r += 32) y[(size_t)e * BS + r] = tmp[warp][r];
    } else {
      for (int r = lane; r < BS; r += 32) {
        const double* A = Uinv + (size_t)e * BS * BS + (size_t)r * BS;
        double s = 0.0;
        for (int m = 0; m < BS; ++m) s += A[m] * tmp[warp][m];
        y[(size_t)e * BS + r] = s;
      }
    }
  }
}

// ------------------------------------------------------------- reductions
// partial[j * nblocks + b] = sum over block b's rows of V_j . w (V_j = V + j*ld)
__global__ void mdot_partial_kernel(long long n, const double* __restrict__ V, long long ld, int nvec,
                                    const double* __restrict__ w, double* __restrict__ partial) {
  __shared__ double red[256];
  int j = blockIdx.y;
  const double* v = V + (size_t)j * ld;
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += v[i] * w[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[(size_t)j * gridDim.x + blockIdx.x] = red[0];
}

__global__ void mdot_final_kernel(int nblocks, int nvec, const double* __restrict__ partial, double* __restrict__ out) {
  __shared__ double red[256];
  int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[(size_t)j * nblocks + b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0];
}

// w += sign * sum_j h[j] V_j
__global__ void maxpy_kernel(long long n, const double* __restrict__ V, long long ld, int nvec,
                             const double* __restrict__ h, double sign, double* __restrict__ w) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < nvec; ++j) s += h[j] * V[(size_t)j * ld + i];
    w[i] += sign * s;
  }
}

// y = a x + b y
__global__ void axpby_kernel(long long n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// z = x + a y
__global__ void xpay_kernel(long long n, const double* __restrict__ x, double a, const double* __restrict__ y,
                            double* __restrict__ z) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = x[i] + a * y[i];
}

// ------------------------------------------------------------- launchers
static int grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 148 * 8 ? (g < 1 ? 1 : g) : 148 * 8);
}

cudaError_t la_mdot(LinalgWork& w, long long n, const double* V, long long ld, int nvec, const double* x,
                    double* d_out, cudaStream_t s) {
  int nb = 148 * 2;
  dim3 grid(nb, nvec);
  mdot_partial_kernel<<<grid, 256, 0, s>>>(n, V, ld, nvec, x, w.partial);
  mdot_final_kernel<<<nvec, 256, 0, s>>>(nb, nvec, w.partial, d_out);
  return cudaGetLastError();
}

cudaError_t la_maxpy(long long n, const double* V, long long ld, int nvec, const double* d_h, double sign, double* w,
                     cudaStream_t s) {
  maxpy_kernel<<<grid_for(n), 256, 0, s>>>(n, V, ld, nvec, d_h, sign, w);
  return cudaGetLastError();
}

cudaError_t la_axpby(long long n, double a, const double* x, double b, double* y, cudaStream_t s) {
  axpby_kernel<<<grid_for(n), 256, 0, s>>>(n, a, x, b, y);
  return cudaGetLastError();
}

cudaError_t la_xpay(long long n, const double* x, double a, const double* y, double* z, cudaStream_t s) {
  xpay_kernel<<<grid_for(n), 256, 0, s>>>(n, x, a, y, z);
  return cudaGetLastError();
}

cudaError_t la_block_invert(int nblk, int bs, const double* src, const int* blk_index, double* dst, int* flag,
                            cudaStream_t s) {
  size_t smem = sizeof(double) * bs * bs + sizeof(int) * bs;
  static size_t attr = 0;
  if (smem > 48 * 1024 && smem > attr) {
    cudaError_t e = cudaFuncSetAttribute(block_invert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = smem;
  }
  block_invert_kernel<<<nblk, 256, smem, s>>>(nblk, bs, src, blk_index, dst, flag);
  return cudaGetLastError();
}

#define ICX_BS_SWITCH(bs, CALL) \
  switch (bs) {                 \
    case 4: { constexpr int B = 4; CALL; } break;     \
    case 9: { constexpr int B = 9; CALL; } break;     \
    case 16: { constexpr int B = 16; CALL; } break;   \
    case 25: { constexpr int B = 25; CALL; } break;   \
    case 36: { constexpr int B = 36; CALL; } break;   \
    case 64: { constexpr int B = 64; CALL; } break;   \
    case 100: { constexpr int B = 100; CALL; } break; \
    default: return cudaErrorInvalidValue;            \
  }

cudaError_t la_block_diag_apply(int E, int bs, const double* D, const double* x, double* y, cudaStream_t s) {
  int blocks = (E + 7) / 8;
  ICX_BS_SWITCH(bs, (block_diag_apply_kernel<B><<<blocks, 256, 0, s>>>(E, D, x, y)));
  return cudaGetLastError();
}

static int level_rows(int nx, int ny, int level) {
  int i0 = level - (ny - 1) > 0 ? level - (ny - 1) : 0;
  int i1 = level < nx - 1 ? level : nx - 1;
  return i1 - i0 + 1;
}

cudaError_t la_ilu_factor(const DeviceMesh& dm, int nx, int ny, double* LU, double* Uinv, int* flag, cudaStream_t s) {
  int bs = dm.nb * dm.neq;
  size_t smem = sizeof(double) * 2 * bs * bs + sizeof(int) * bs;
  static size_t attr = 0;
  if (smem > 48 * 1024 && smem > attr) {
    cudaError_t e = cudaFuncSetAttribute(ilu_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = smem;
  }
  for (int level = 0; level < nx + ny - 1; ++level)
    ilu_level_kernel<<<level_rows(nx, ny, level), 256, smem, s>>>(nx, ny, level, bs, dm.bsr_rowptr, dm.bsr_colidx,
                                                                  LU, Uinv, flag);
  return cudaGetLastError();
}

cudaError_t la_ilu_apply(const DeviceMesh& dm, int nx, int ny, const double* LU, const double* Uinv, const double* x,
                         double* y, cudaStream_t s) {
  int bs = dm.nb * dm.neq;
  for (int pass = 0; pass < 2; ++pass) {
    int fwd = pass == 0;
    for (int l = 0; l < nx + ny - 1; ++l) {
      int level = fwd ? l : nx + ny - 2 - l;
      int blocks = (level_rows(nx, ny, level) + 3) / 4;
      ICX_BS_SWITCH(bs, (ilu_solve_level_kernel<B><<<blocks, 128, 0, s>>>(nx, ny, level, fwd, dm.bsr_rowptr,
                                                                           dm.bsr_colidx, LU, Uinv, x, y)));
    }
  }
  return cudaGetLastError();
}

}  // namespace icx

// ------------------------------------------------------------------ GMRES
namespace icx {

double la_norm(LinalgWork& lw, long long n, const double* x, double* d_scratch, cudaStream_t s) {
  la_mdot(lw, n, x, 0, 1, x, d_scratch, s);
  double h = 0.0;
  cudaMemcpyAsync(&h, d_scratch, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return std::sqrt(h);
}

#define GCK(expr)                                                  \
  do {                                                             \
    cudaError_t _e = (expr);                                       \
    if (_e != cudaSuccess) {                                       \
      if (err) *err = std::string(#expr) + ": " + cudaGetErrorString(_e); \
      return ICX_ERR_CUDA;                                         \
    }                                                              \
  } while (0)

icx_status gmres_op(KrylovBuffers& kb, const LinOp& A, const LinOp* M, int maxit, double rtol, const double* b,
                    double* x, int* iters, double* relres, cudaStream_t s, std::string* err) {
  long long n = kb.n;
  int m = kb.m;
  if (b == kb.r || b == kb.w || b == kb.z || x == kb.r || x == kb.w || x == kb.z) {
    if (err) *err = "gmres vectors alias its work buffers";
    return ICX_ERR_INVALID;
  }
  GCK(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
  double bnorm = la_norm(*kb.lw, n, b, kb.dh, s);
  *iters = 0;
  *relres = 0.0;
  if (bnorm == 0.0) return ICX_OK;
  if (!std::isfinite(bnorm)) {
    if (err) *err = "non-finite right-hand side";
    return ICX_ERR_NONFINITE;
  }
  double tol = rtol * bnorm;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hcol(m + 2), hp(m + 1);
  GCK(cudaMemcpyAsync(kb.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  double beta = bnorm;
  int total = 0;
  while (true) {
    GCK(la_axpby(n, 1.0 / beta, kb.r, 0.0, kb.V, s));
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    double resid = beta;
    for (; j < m && total < maxit; ++j) {
      double* vj = kb.V + (size_t)j * n;
      double* vj1 = kb.V + (size_t)(j + 1) * n;
      if (M) {
        GCK((*M)(vj, kb.z));
        GCK(A(kb.z, vj1));
      } else {
        GCK(A(vj, vj1));
      }
      // classical Gram-Schmidt, twice
      std::fill(hcol.begin(), hcol.end(), 0.0);
      for (int pass = 0; pass < 2; ++pass) {
        GCK(la_mdot(*kb.lw, n, kb.V, n, j + 1, vj1, kb.dh, s));
        GCK(la_maxpy(n, kb.V, n, j + 1, kb.dh, -1.0, vj1, s));
        GCK(cudaMemcpyAsync(hp.data(), kb.dh, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
        GCK(cudaStreamSynchronize(s));
        for (int i = 0; i <= j; ++i) hcol[i] += hp[i];
      }
      double hn = la_norm(*kb.lw, n, vj1, kb.dh, s);
      hcol[j + 1] = hn;
      if (!std::isfinite(hn)) {
        if (err) *err = "non-finite Krylov vector";
        return ICX_ERR_NONFINITE;
      }
      if (hn > 0.0) GCK(la_axpby(n, 1.0 / hn, vj1, 0.0, vj1, s));
      for (int i = 0; i < j; ++i) {
        double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
        hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
        hcol[i] = t;
      }
      double den = std::hypot(hcol[j], hcol[j + 1]);
      cs[j] = den == 0.0 ? 1.0 : hcol[j] / den;
      sn[j] = den == 0.0 ? 0.0 : hcol[j + 1] / den;
      hcol[j] = den;
      hcol[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hcol[i];
      ++total;
      resid = std::fabs(g[j + 1]);
      if (resid <= tol || hn == 0.0) { ++j; break; }
    }
    for (int i = j - 1; i >= 0; --i) {
      double sacc = g[i];
      for (int k = i + 1; k < j; ++k) sacc -= H[(size_t)i * m + k] * y[k];
      y[i] = sacc / H[(size_t)i * m + i];
    }
    GCK(cudaMemcpyAsync(kb.dh, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, s));
    GCK(cudaMemsetAsync(kb.w, 0, sizeof(double) * n, s));
    GCK(la_maxpy(n, kb.V, n, j, kb.dh, 1.0, kb.w, s));
    if (M) {
      GCK((*M)(kb.w, kb.z));
      GCK(la_axpby(n, 1.0, kb.z, 1.0, x, s));
    } else {
      GCK(la_axpby(n, 1.0, kb.w, 1.0, x, s));
    }
    GCK(A(x, kb.w));
    GCK(la_xpay(n, b, -1.0, kb.w, kb.r, s));
    beta = la_norm(*kb.lw, n, kb.r, kb.dh, s);
    *relres = beta / bnorm;
    if (beta <= tol || total >= maxit || resid <= tol) break;
  }
  *iters = total;
  return ICX_OK;
}

}  // namespace icx
