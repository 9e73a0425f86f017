// Device linear algebra for the Newton solver: block-diagonal inversion
// (block-Jacobi preconditioner), block-ILU(0) on the element block pattern,
// deterministic reductions and the multi-vector kernels of GMRES.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "icx_internal.h"
#include "icx_linalg.h"
#include "icx_blockrow.cuh"
#include "icx_blockinv.cuh"
#include "icx_ilu_rows.cuh"

namespace icx {

// ----------------------------------------------------- block inversion
// gj_invert / write_inverse / InvSmem: icx_blockinv.cuh

// inverse of one diagonal block per CTA; a singular block becomes the
// identity and raises *flag (the preconditioner degrades to no-op on it)
template <int BS>
__global__ void __launch_bounds__(256) block_invert_kernel(int nblk, const double* __restrict__ src,
                                                           const int* __restrict__ blk_index,
                                                           double* __restrict__ dst, int* flag) {
  extern __shared__ double sh[];
  double* a = sh;
  double* fcol = a + BS * BS;
  int* perm = reinterpret_cast<int*>(fcol + BS);
  int* colsrc = perm + BS;
  __shared__ int singular;
  int b = blockIdx.x;
  if (b >= nblk) return;
  const double* A = src + (size_t)blk_index[b] * BS * BS;
  for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) a[t] = A[t];
  __syncthreads();
  gj_invert<BS>(a, perm, fcol, &singular);
  __syncthreads();
  if (singular && threadIdx.x == 0) atomicExch(flag, 1);
  write_inverse<BS>(a, perm, colsrc, singular, dst + (size_t)b * BS * BS);
}

// ------------------------------------------------------------ block-ILU(0)
// Block ILU(0) on the element block pattern in natural (element) order, IKJ
// form: for each row e, for each lower block (e, k) in ascending k,
//   A_ek <- A_ek inv(A_kk);  A_ej -= A_ek A_kj  for every (k, j), j > k, with (e, j) in the pattern;
// then inv(A_ee) is stored for the next rows and the backward solve. On the
// structured element grid row (i, j) depends only on (i-1, j) and (i, j-1),
// so the rows of one anti-diagonal i + j = level are independent (in a batch
// of grids, the rows of that level in every grid): one launch per level, one
// CTA per row.

__device__ inline int find_block(const int* rowptr, const int* colidx, int r, int c) {
  for (int k = rowptr[r]; k < rowptr[r + 1]; ++k)
    if (colidx[k] == c) return k;
  return -1;
}

// C = X Y for BS x BS blocks in shared memory, each thread owning 4 x 4
// output tiles; op(tile, r0, c0, acc) consumes every finished tile
template <int BS, class Op>
__device__ inline void block_gemm(const double* X, const double* Y, Op op) {
  constexpr int NT = (BS + 3) / 4;
  for (int tt = threadIdx.x; tt < NT * NT; tt += blockDim.x) {
    const int r0 = (tt / NT) * 4, c0 = (tt % NT) * 4;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int m = 0; m < BS; ++m) {
      double xa[4], yb[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) xa[a] = (r0 + a < BS) ? X[(r0 + a) * BS + m] : 0.0;
      if (BS % 4 == 0) {
        const double2* y2 = reinterpret_cast<const double2*>(Y + m * BS + c0);
        double2 u0 = y2[0], u1 = y2[1];
        yb[0] = u0.x; yb[1] = u0.y; yb[2] = u1.x; yb[3] = u1.y;
      } else {
#pragma unroll
        for (int b = 0; b < 4; ++b) yb[b] = (c0 + b < BS) ? Y[m * BS + c0 + b] : 0.0;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += xa[a] * yb[b];
    }
    op(r0, c0, acc);
  }
}

template <int BS>
struct IluSmem {
  static constexpr size_t BYTES = sizeof(double) * (2 * BS * BS + BS) + sizeof(int) * 2 * BS;
};

template <int BS>
__global__ void __launch_bounds__(256) ilu_level_kernel(int E, int nnzb, const int* __restrict__ elems,
                                                        const int* __restrict__ rowptr,
                                                        const int* __restrict__ colidx, double* __restrict__ LU,
                                                        double* __restrict__ Uinv, int* flag) {
  extern __shared__ double sh[];
  double* X = sh;                  // BS x BS
  double* Y = X + BS * BS;         // BS x BS
  double* fcol = Y + BS * BS;      // BS
  int* perm = reinterpret_cast<int*>(fcol + BS);
  int* colsrc = perm + BS;
  __shared__ int singular;
  const int e = elems[blockIdx.x];
  // block and element indices are checked before use: a bad one sets
  // *flag = 2 and the CTA leaves (the values are uniform over the CTA)
  if (e < 0 || e >= E || rowptr[e] < 0 || rowptr[e + 1] > nnzb) {
    if (threadIdx.x == 0) atomicExch(flag, 2);
    return;
  }
  for (int kl = rowptr[e]; kl < rowptr[e + 1]; ++kl) {
    const int k = colidx[kl];
    if (k < 0 || k >= E) {
      if (threadIdx.x == 0) atomicExch(flag, 2);
      return;
    }
    if (k >= e) break;  // columns ascend: the lower blocks come first
    double* Aek = LU + (size_t)kl * BS * BS;
    const double* Ui = Uinv + (size_t)k * BS * BS;
    __syncthreads();
    for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) {
      X[t] = Aek[t];
      Y[t] = Ui[t];
    }
    __syncthreads();
    // L_ek = A_ek inv(U_kk): kept in registers until every thread has read X
    constexpr int NT = (BS + 3) / 4;
    constexpr int MAXT = (NT * NT + 255) / 256;
    double keep[MAXT][4][4];
    int slot = 0;
    block_gemm<BS>(X, Y, [&](int r0, int c0, double (&acc)[4][4]) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) keep[slot][a][b] = acc[a][b];
      ++slot;
    });
    __syncthreads();
    slot = 0;
    for (int tt = threadIdx.x; tt < NT * NT; tt += blockDim.x, ++slot) {
      const int r0 = (tt / NT) * 4, c0 = (tt % NT) * 4;
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
          if (r0 + a < BS && c0 + b < BS) {
            X[(r0 + a) * BS + c0 + b] = keep[slot][a][b];
            Aek[(r0 + a) * BS + c0 + b] = keep[slot][a][b];
          }
    }
    // A_ej -= L_ek U_kj for the upper blocks of row k that lie in row e's pattern
    for (int kj = rowptr[k]; kj < rowptr[k + 1]; ++kj) {
      const int jc = colidx[kj];
      if (jc <= k) continue;
      const int ej = find_block(rowptr, colidx, e, jc);
      if (ej < 0) continue;  // outside the pattern: dropped (level 0 fill)
      if (kj >= nnzb || ej >= nnzb) {
        if (threadIdx.x == 0) atomicExch(flag, 2);
        return;
      }
      const double* Akj = LU + (size_t)kj * BS * BS;
      double* Aej = LU + (size_t)ej * BS * BS;
      __syncthreads();
      for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) Y[t] = Akj[t];
      __syncthreads();
      block_gemm<BS>(X, Y, [&](int r0, int c0, double (&acc)[4][4]) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b)
            if (r0 + a < BS && c0 + b < BS) Aej[(r0 + a) * BS + c0 + b] -= acc[a][b];
      });
    }
  }
  __syncthreads();
  const int kd = find_block(rowptr, colidx, e, e);
  if (kd < 0) {
    if (threadIdx.x == 0) atomicExch(flag, 2);
    return;
  }
  const double* Aee = LU + (size_t)kd * BS * BS;
  for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) X[t] = Aee[t];
  __syncthreads();
  gj_invert<BS>(X, perm, fcol, &singular);
  __syncthreads();
  if (singular && threadIdx.x == 0) atomicExch(flag, 1);
  write_inverse<BS>(X, perm, colsrc, singular, Uinv + (size_t)e * BS * BS);
}

// After the factorisation every upper block is scaled by the inverse of its
// row's diagonal block, U_ek <- inv(U_ee) U_ek (k > e), so that the backward
// substitution y_e = inv(U_ee) (f_e - sum_{k>e} U_ek y_k) becomes
//   y_e = inv(U_ee) f_e - sum_{k>e} (inv(U_ee) U_ek) y_k,
// a plain block-row product whose rows can be split across warps.
// One CTA per row, both operands staged in shared memory.
template <int BS>
__global__ void __launch_bounds__(256) ilu_scale_upper_kernel(int E, const int* __restrict__ rowptr,
                                                              const int* __restrict__ colidx,
                                                              double* __restrict__ LU,
                                                              const double* __restrict__ Uinv) {
  extern __shared__ double sh[];
  double* D = sh;            // BS x BS
  double* B = sh + BS * BS;  // BS x BS
  const int e = blockIdx.x;
  if (e >= E) return;
  const double* Di = Uinv + (size_t)e * BS * BS;
  for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) D[t] = Di[t];
  for (int kb = rowptr[e]; kb < rowptr[e + 1]; ++kb) {
    if (colidx[kb] <= e) continue;
    double* U = LU + (size_t)kb * BS * BS;
    __syncthreads();
    for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) B[t] = U[t];
    __syncthreads();
    block_gemm<BS>(D, B, [&](int r0, int c0, double (&acc)[4][4]) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
          if (r0 + a < BS && c0 + b < BS) U[(r0 + a) * BS + c0 + b] = acc[a][b];
    });
  }
}

// ------------------------------------------------------------- reductions
// partial[j * nblocks + b] = sum over block b's rows of V_j . x (V_j = V + j*ld;
// an FP32 basis is widened to FP64 before the product), G vectors per pass
// over x: each thread holds x_i once per group of G basis vectors, so x is
// read ceil(nvec / G) times instead of nvec times (the vectors V_j once
// each); per block the sums are reduced by shuffles, then across the warps in
// a fixed order
template <class TV, int G>
__global__ void __launch_bounds__(256) mdot_grouped_kernel(long long n, const TV* __restrict__ V, long long ld,
                                                           int nvec, const double* __restrict__ x,
                                                           double* __restrict__ partial) {
  __shared__ double red[G][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j0 = 0; j0 < nvec; j0 += G) {
    double acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
      const double xi = x[i];
#pragma unroll
      for (int g = 0; g < G; ++g)
        if (j0 + g < nvec) acc[g] += (double)V[(size_t)(j0 + g) * ld + i] * xi;
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      double v = acc[g];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) red[g][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < G && j0 + (int)threadIdx.x < nvec) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) s += red[threadIdx.x][w];
      partial[(size_t)(j0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
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
template <class TV>
__global__ void maxpy_kernel(long long n, const TV* __restrict__ V, long long ld, int nvec,
                             const double* __restrict__ h, double sign, double* __restrict__ w) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < nvec; ++j) s += h[j] * (double)V[(size_t)j * ld + i];
    w[i] += sign * s;
  }
}

// v32 = a x rounded to FP32
__global__ void scale_to_f32_kernel(long long n, double a, const double* __restrict__ x, float* __restrict__ v32) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v32[i] = (float)(a * x[i]);
}

// v32 = w / sqrt(*h2) rounded to FP32 (w itself when *h2 is not positive)
__global__ void normalize_to_f32_kernel(long long n, const double* __restrict__ h2, const double* __restrict__ w,
                                        float* __restrict__ v32) {
  const double h = *h2;
  const double a = h > 0.0 ? 1.0 / sqrt(h) : 1.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v32[i] = (float)(a * w[i]);
}

// y = a x + b y
__device__ inline double axpby_val(double a, double x, double b, double y) { return a * x + b * y; }

__global__ void axpby_kernel(long long n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = axpby_val(a, x[i], b, y[i]);
}

// v /= sqrt(*h2) when *h2 > 0, with the same operations as
// la_axpby(n, 1 / sqrt(h2), v, 0, v) after the host has read h2
__global__ void normalize_kernel(long long n, const double* __restrict__ h2, double* v) {
  const double h = *h2;
  if (!(h > 0.0)) return;
  const double a = 1.0 / sqrt(h);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = axpby_val(a, v[i], 0.0, v[i]);
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
  const int nb = kMdotBlocks;
  mdot_grouped_kernel<double, 8><<<nb, 256, 0, s>>>(n, V, ld, nvec, x, w.partial);
  mdot_final_kernel<<<nvec, 256, 0, s>>>(nb, nvec, w.partial, d_out);
  return cudaGetLastError();
}

cudaError_t la_mdot32(LinalgWork& w, long long n, const float* V, long long ld, int nvec, const double* x,
                      double* d_out, cudaStream_t s) {
  const int nb = kMdotBlocks;
  mdot_grouped_kernel<float, 8><<<nb, 256, 0, s>>>(n, V, ld, nvec, x, w.partial);
  mdot_final_kernel<<<nvec, 256, 0, s>>>(nb, nvec, w.partial, d_out);
  return cudaGetLastError();
}

cudaError_t la_maxpy(long long n, const double* V, long long ld, int nvec, const double* d_h, double sign, double* w,
                     cudaStream_t s) {
  maxpy_kernel<double><<<grid_for(n), 256, 0, s>>>(n, V, ld, nvec, d_h, sign, w);
  return cudaGetLastError();
}

cudaError_t la_maxpy32(long long n, const float* V, long long ld, int nvec, const double* d_h, double sign, double* w,
                       cudaStream_t s) {
  maxpy_kernel<float><<<grid_for(n), 256, 0, s>>>(n, V, ld, nvec, d_h, sign, w);
  return cudaGetLastError();
}

// matrix-free products: slot = {|v|^2, c}, h = c / |v| (c when v = 0)
__device__ inline double fd_step(const double* slot) {
  const double v2 = slot[0];
  return v2 > 0.0 ? slot[1] / sqrt(v2) : slot[1];
}

__global__ void fd_perturb_kernel(long long n, const double* __restrict__ u, const double* __restrict__ v,
                                  const double* __restrict__ slot, double* __restrict__ up) {
  const double h = fd_step(slot);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    up[i] = u[i] + h * v[i];
}

__global__ void fd_diff_kernel(long long n, const double* __restrict__ rp, const double* __restrict__ r0,
                               const double* __restrict__ slot, double* __restrict__ y) {
  const double h = fd_step(slot);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = (rp[i] - r0[i]) / h;
}

cudaError_t la_fd_perturb(long long n, const double* u, const double* v, const double* slot, double* up,
                          cudaStream_t s) {
  fd_perturb_kernel<<<grid_for(n), 256, 0, s>>>(n, u, v, slot, up);
  return cudaGetLastError();
}

cudaError_t la_fd_diff(long long n, const double* rp, const double* r0, const double* slot, double* y,
                       cudaStream_t s) {
  fd_diff_kernel<<<grid_for(n), 256, 0, s>>>(n, rp, r0, slot, y);
  return cudaGetLastError();
}

__global__ void scale_kernel(long long n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i];
}

cudaError_t la_scale(long long n, double a, const double* x, double* y, cudaStream_t s) {
  scale_kernel<<<grid_for(n), 256, 0, s>>>(n, a, x, y);
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

template <class K>
static cudaError_t smem_attr(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t la_block_invert(int nblk, int bs, const double* src, const int* blk_index, double* dst, int* flag,
                            cudaStream_t s) {
#define ICX_INV_CASE(B)                                                                        \
  if (bs == B) {                                                                               \
    cudaError_t e = smem_attr(block_invert_kernel<B>, InvSmem<B>::BYTES);                      \
    if (e != cudaSuccess) return e;                                                            \
    block_invert_kernel<B><<<nblk, 256, InvSmem<B>::BYTES, s>>>(nblk, src, blk_index, dst, flag); \
    return cudaGetLastError();                                                                 \
  }
  ICX_BLOCK_SIZES(ICX_INV_CASE)
#undef ICX_INV_CASE
  return cudaErrorInvalidValue;
}

template <class TA>
static cudaError_t tri_rows_t(const DeviceMesh& dm, bool lower, const TA* A, const double* v, const double* x0,
                              double sign, double* y, cudaStream_t s) {
  const int bs = dm.nb * dm.neq;
  RowSet rs{0, 0, -1, dm.E};
#define ICX_TRI_CASE(B)                                                                                          \
  if (bs == B)                                                                                                   \
    return lower ? launch_block_rows<B, BR_LOWER, TA>(rs, dm.bsr_rowptr, dm.bsr_colidx, A, v, x0, sign, y, s)    \
                 : launch_block_rows<B, BR_UPPER, TA>(rs, dm.bsr_rowptr, dm.bsr_colidx, A, v, x0, sign, y, s);
  ICX_BLOCK_SIZES(ICX_TRI_CASE)
#undef ICX_TRI_CASE
  return cudaErrorInvalidValue;
}

cudaError_t la_tri_rows(const DeviceMesh& dm, bool lower, const double* A, const double* v, const double* x0,
                        double sign, double* y, cudaStream_t s) {
  return tri_rows_t<double>(dm, lower, A, v, x0, sign, y, s);
}
cudaError_t la_tri_rows_f32(const DeviceMesh& dm, bool lower, const float* A, const double* v, const double* x0,
                            double sign, double* y, cudaStream_t s) {
  return tri_rows_t<float>(dm, lower, A, v, x0, sign, y, s);
}

cudaError_t la_block_diag_apply(int E, int bs, const double* D, const double* x, double* y, cudaStream_t s) {
  RowSet rs{0, 0, -1, E};
#define ICX_DIAG_CASE(B) \
  if (bs == B) return launch_block_rows<B, BR_DIAG>(rs, nullptr, nullptr, D, x, nullptr, 1.0, y, s);
  ICX_BLOCK_SIZES(ICX_DIAG_CASE)
#undef ICX_DIAG_CASE
  return cudaErrorInvalidValue;
}


cudaError_t la_ilu_factor(const DeviceMesh& dm, const int* order, const std::vector<int>& lvl_off, double* LU,
                          double* Uinv, int* flag, cudaStream_t s) {
  const int bs = dm.nb * dm.neq;
#define ICX_ILUF_CASE(B)                                                                               \
  if (bs == B) {                                                                                       \
    cudaError_t e = smem_attr(ilu_level_kernel<B>, IluSmem<B>::BYTES);                                 \
    if (e == cudaSuccess) e = smem_attr(ilu_scale_upper_kernel<B>, IluSmem<B>::BYTES);                 \
    if (e != cudaSuccess) return e;                                                                    \
    for (size_t l = 0; l + 1 < lvl_off.size(); ++l) {                                                  \
      const int cnt = lvl_off[l + 1] - lvl_off[l];                                                     \
      if (cnt > 0)                                                                                     \
        ilu_level_kernel<B><<<cnt, 256, IluSmem<B>::BYTES, s>>>(dm.E, dm.nnzb, order + lvl_off[l],     \
                                                                dm.bsr_rowptr, dm.bsr_colidx, LU, Uinv, flag); \
    }                                                                                                  \
    ilu_scale_upper_kernel<B><<<dm.E, 256, IluSmem<B>::BYTES, s>>>(dm.E, dm.bsr_rowptr, dm.bsr_colidx, LU, Uinv); \
    return cudaGetLastError();                                                                         \
  }
  ICX_BLOCK_SIZES(ICX_ILUF_CASE)
#undef ICX_ILUF_CASE
  return cudaErrorInvalidValue;
}

// rows per task compiled for a block size: at most the block size, and the
// three blocks' rows a task holds (R x column chunks each) at most 24 values
// per lane, which keeps them in registers

template <int B, int R, class TA>
static const void* flow_kernel_if_fit(bool sen) {
  if constexpr (flow_rows_fit(B, (B + 31) / 32, R))
    return sen ? (const void*)ilu_apply_flow_kernel<B, R, TA, true> : (const void*)ilu_apply_flow_kernel<B, R, TA, false>;
  else return nullptr;
}

// the data-flow kernel for `rows` rows per task (0: the default) on the
// counter or the sentinel schedule, or null
template <int B, class TA>
static const void* flow_kernel_for(int rows, bool sen) {
  static_assert(kFlowRows[0] == 2 && kFlowRows[1] == 4 && kFlowRows[2] == 6 && kFlowRows[3] == 8, "tiles");
  switch (rows ? rows : FlowCfg<B>::R_DEFAULT) {
    case 2: return flow_kernel_if_fit<B, 2, TA>(sen);
    case 4: return flow_kernel_if_fit<B, 4, TA>(sen);
    case 6: return flow_kernel_if_fit<B, 6, TA>(sen);
    case 8: return flow_kernel_if_fit<B, 8, TA>(sen);
    default: return nullptr;
  }
}

__global__ void flow_fill_kernel(long long n, double* __restrict__ f, double* __restrict__ y) {
  const double v = __longlong_as_double((long long)FLOW_SENTINEL);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    f[i] = v;
    y[i] = v;
  }
}

template <class TA>
static cudaError_t ilu_apply_flow_t(const DeviceMesh& dm, const int* order, const TA* LU,
                                   const TA* Uinv, const double* x, double* y, double* f, unsigned* cnt_f,
                                   unsigned* cnt_b, unsigned epoch, int* err, cudaStream_t s) {
  const int bs = dm.nb * dm.neq;
  int dev = 0, nsm = 0, coop = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (e != cudaSuccess) return e;
  if (!coop) return cudaErrorNotSupported;
  IluFlowArgs<TA> args{dm.E, dm.nnzb, dm.bsr_rowptr, dm.bsr_colidx, dm.bsr_diag, order, LU, Uinv, x, f, y, cnt_f,
                       cnt_b, epoch, err};
  const int pi = sizeof(TA) == 8 ? 0 : 1;
  const int rows = dm.tile.flow_rows[pi], ctas = dm.tile.flow_ctas[pi];
  if (ctas < 0) return cudaErrorInvalidValue;
  const bool sen = flow_sentinel(dm.tile, pi);
  const void* kern = nullptr;
#define ICX_ILUF2_CASE(B)                                                                  \
  if (bs == B) kern = flow_kernel_for<B, TA>(rows, sen);
  ICX_BLOCK_SIZES(ICX_ILUF2_CASE)
#undef ICX_ILUF2_CASE
  if (!kern) return cudaErrorInvalidValue;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorNotSupported;
  // the whole grid is resident (the tasks wait on one another): at most the
  // occupancy limit per SM; two by default
  const int want = ctas ? ctas : 2;
  const int grid = nsm * (per_sm < want ? per_sm : want);
  if (sen) {
    const long long n = (long long)dm.E * bs;
    flow_fill_kernel<<<grid_for(n), 256, 0, s>>>(n, f, y);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(256), params, 0, s);
}

int flow_rows_default(int bs) {
#define ICX_FLOWR_CASE(B) \
  if (bs == B) return FlowCfg<B>::R_DEFAULT;
  ICX_BLOCK_SIZES(ICX_FLOWR_CASE)
#undef ICX_FLOWR_CASE
  return 0;
}

bool flow_rows_compiled(int bs, int rows) {
  if (rows == 0) return true;
  const int ns = (bs + 31) / 32;
  for (int r : kFlowRows)
    if (r == rows) return flow_rows_fit(bs, ns, r);
  return false;
}

template <class TA>
static cudaError_t ilu_apply_rows_t(const DeviceMesh& dm, int nx, int ny, const TA* LU, const TA* Uinv,
                                   const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b,
                                   unsigned epoch, int* err, cudaStream_t s) {
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (nx < 1 || ny < 1 || nx * ny != dm.E) return cudaErrorInvalidValue;
  const int bs = dm.nb * dm.neq;
  IluRowArgs<TA> a{nx, ny, dm.nnzb, dm.bsr_rowptr, dm.bsr_colidx, dm.bsr_diag, LU, Uinv, x, f, y, cnt_f, cnt_b,
                   epoch, err};
  void* params[] = {&a};
#define ICX_ROWS_CASE(B)                                                                              \
  if (bs == B) {                                                                                      \
    using K = IluRowCfg<B, TA>;                                                                       \
    if ((e = smem_attr(ilu_apply_rows_kernel<B, TA>, K::SMEM)) != cudaSuccess) return e;              \
    int per_sm = 0;                                                                                   \
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ilu_apply_rows_kernel<B, TA>, 128, K::SMEM); \
    if (e != cudaSuccess) return e;                                                                   \
    if ((long long)per_sm * nsm < ny) return cudaErrorNotSupported;                                   \
    return cudaLaunchCooperativeKernel((const void*)ilu_apply_rows_kernel<B, TA>, dim3(ny), dim3(128), params, \
                                       K::SMEM, s);                                                   \
  }
  ICX_ROWS_CASE(4) ICX_ROWS_CASE(9) ICX_ROWS_CASE(16) ICX_ROWS_CASE(25) ICX_ROWS_CASE(36) ICX_ROWS_CASE(64)
#undef ICX_ROWS_CASE
  return cudaErrorNotSupported;
}

cudaError_t la_ilu_apply_rows(const DeviceMesh& dm, int nx, int ny, const double* LU, const double* Uinv,
                              const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b, unsigned epoch,
                              int* err, cudaStream_t s) {
  return ilu_apply_rows_t<double>(dm, nx, ny, LU, Uinv, x, y, f, cnt_f, cnt_b, epoch, err, s);
}

cudaError_t la_ilu_apply_rows_f32(const DeviceMesh& dm, int nx, int ny, const float* LU, const float* Uinv,
                                  const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b,
                                  unsigned epoch, int* err, cudaStream_t s) {
  return ilu_apply_rows_t<float>(dm, nx, ny, LU, Uinv, x, y, f, cnt_f, cnt_b, epoch, err, s);
}

cudaError_t la_ilu_apply_flow(const DeviceMesh& dm, const int* order, const double* LU, const double* Uinv,
                              const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b, unsigned epoch,
                              int* err, cudaStream_t s) {
  return ilu_apply_flow_t<double>(dm, order, LU, Uinv, x, y, f, cnt_f, cnt_b, epoch, err, s);
}

cudaError_t la_ilu_apply_flow_f32(const DeviceMesh& dm, const int* order, const float* LU, const float* Uinv,
                                  const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b,
                                  unsigned epoch, int* err, cudaStream_t s) {
  return ilu_apply_flow_t<float>(dm, order, LU, Uinv, x, y, f, cnt_f, cnt_b, epoch, err, s);
}

cudaError_t la_block_diag_correct_f32(int E, int bs, const float* D, const double* y, double* z, cudaStream_t s) {
  RowSet rs{0, 0, -1, E};
#define ICX_CORR_CASE(B) \
  if (bs == B) return launch_block_rows<B, BR_DIAG, float>(rs, nullptr, nullptr, D, y, y, 1.0, z, s);
  ICX_BLOCK_SIZES(ICX_CORR_CASE)
#undef ICX_CORR_CASE
  return cudaErrorInvalidValue;
}

__global__ void dot_to_kernel(long long n, const double* __restrict__ x, const double* __restrict__ y,
                              double* __restrict__ out) {
  __shared__ double red[256];
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

cudaError_t la_dot_to(long long n, const double* x, const double* y, double* d_out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  dot_to_kernel<<<592, 256, 0, s>>>(n, x, y, d_out);
  return cudaGetLastError();
}

cudaError_t la_block_diag_apply_f32(int E, int bs, const float* D, const double* x, double* y, cudaStream_t s) {
  RowSet rs{0, 0, -1, E};
#define ICX_DIAG32_CASE(B) \
  if (bs == B) return launch_block_rows<B, BR_DIAG, float>(rs, nullptr, nullptr, D, x, nullptr, 1.0, y, s);
  ICX_BLOCK_SIZES(ICX_DIAG32_CASE)
#undef ICX_DIAG32_CASE
  return cudaErrorInvalidValue;
}

__global__ void d2f_kernel(long long n, const double* __restrict__ x, float* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

cudaError_t la_d2f(long long n, const double* x, float* y, cudaStream_t s) {
  d2f_kernel<<<grid_for(n), 256, 0, s>>>(n, x, y);
  return cudaGetLastError();
}

__global__ void d2bf_kernel(long long n, const double* __restrict__ x, __nv_bfloat16* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __double2bfloat16(x[i]);
}

cudaError_t la_d2bf(long long n, const double* x, __nv_bfloat16* y, cudaStream_t s) {
  d2bf_kernel<<<grid_for(n), 256, 0, s>>>(n, x, y);
  return cudaGetLastError();
}

__global__ void f2d_kernel(long long n, const float* __restrict__ x, double* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = (double)x[i];
}

cudaError_t la_f2d(long long n, const float* x, double* y, cudaStream_t s) {
  f2d_kernel<<<grid_for(n), 256, 0, s>>>(n, x, y);
  return cudaGetLastError();
}

// dst block b = src block map[b]; each CTA copies whole blocks with 16-byte
// vector loads (a block of bs x bs doubles starts on a 16-byte boundary when
// bs * bs is even; odd sizes fall back to 8-byte copies)
__global__ void gather_blocks_kernel(int nblk, int bs2, const double* __restrict__ src, const int* __restrict__ map,
                                     double* __restrict__ dst) {
  for (int b = blockIdx.x; b < nblk; b += gridDim.x) {
    const double* s = src + (size_t)map[b] * bs2;
    double* d = dst + (size_t)b * bs2;
    if ((bs2 & 1) == 0) {
      const double2* s2 = reinterpret_cast<const double2*>(s);
      double2* d2 = reinterpret_cast<double2*>(d);
      for (int t = threadIdx.x; t < bs2 / 2; t += blockDim.x) d2[t] = __ldcs(s2 + t);
    } else {
      for (int t = threadIdx.x; t < bs2; t += blockDim.x) d[t] = __ldcs(s + t);
    }
  }
}

cudaError_t la_gather_blocks(int nblk, int bs, const double* src, const int* map, double* dst, cudaStream_t s) {
  if (nblk <= 0) return cudaSuccess;
  const int grid = nblk < 148 * 16 ? nblk : 148 * 16;
  gather_blocks_kernel<<<grid, 256, 0, s>>>(nblk, bs * bs, src, map, dst);
  return cudaGetLastError();
}

}  // namespace icx

// ------------------------------------------------------------------ GMRES
namespace icx {

double la_norm(LinalgWork& lw, long long n, const double* x, double* d_scratch, cudaStream_t s) {
  // a failed launch or copy gives NaN: callers treat a non-finite norm as an error
  if (la_mdot(lw, n, x, 0, 1, x, d_scratch, s) != cudaSuccess) return NAN;
  double h = 0.0;
  if (cudaMemcpyAsync(&h, d_scratch, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return NAN;
  if (cudaStreamSynchronize(s) != cudaSuccess) return NAN;
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

void ArnoldiGraphs::reset() {
  for (cudaGraphExec_t& g : exec)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  std::fill(seen.begin(), seen.end(), 0);
  failed = false;
}

void ArnoldiGraphs::release() {
  reset();
  exec.clear();
  seen.clear();
  if (cap) cudaStreamDestroy(cap), cap = nullptr;
  if (hp) cudaFreeHost(hp), hp = nullptr;
  for (cudaEvent_t& ev : done)
    if (ev) cudaEventDestroy(ev), ev = nullptr;
  key = 0;
  m = 0;
}

// prepares the graph set for operators `key` and restart length m (drops
// graphs of another key); false when it cannot be used
static bool arnoldi_graphs_ready(ArnoldiGraphs& g, unsigned long long key, int m) {
  if (g.m != m) {
    g.release();
    g.m = m;
    g.exec.assign(m, nullptr);
    g.seen.assign(m, 0);
  }
  if (!g.cap && cudaStreamCreateWithFlags(&g.cap, cudaStreamNonBlocking) != cudaSuccess) return false;
  if (!g.hp && cudaMallocHost((void**)&g.hp, sizeof(double) * 6 * (m + 2)) != cudaSuccess) return false;
  for (cudaEvent_t& ev : g.done)
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return false;
  if (g.key != key) {
    g.reset();
    g.key = key;
  }
  return !g.failed;
}

// the graph of Arnoldi step j: captured on the step's second eager run under
// the current key (the first run has done every one-time setup of the
// kernels it launches), then replayed; it copies its reductions to host
// half j % 2. Null: run the step eagerly.
template <class Step>
static cudaGraphExec_t arnoldi_graph(ArnoldiGraphs& g, int j, long long n, double* vj1, const double* h2, Step& step,
                                     bool append_normalize) {
  if (g.failed) return nullptr;
  if (g.exec[j]) return g.exec[j];
  if (g.seen[j]++ < 1) return nullptr;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(g.cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t es = step(g.cap, g.hp + (size_t)(j & 1) * 3 * (g.m + 2));
    if (es == cudaSuccess && append_normalize) {
      normalize_kernel<<<grid_for(n), 256, 0, g.cap>>>(n, h2, vj1);
      es = cudaGetLastError();
    }
    e = cudaStreamEndCapture(g.cap, &graph);
    if (es != cudaSuccess) e = es;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec[j], graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    // operators that cannot be captured: eager steps from now on under this key
    (void)cudaGetLastError();
    g.exec[j] = nullptr;
    g.failed = true;
    return nullptr;
  }
  return g.exec[j];
}

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
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hcol(m + 2), hp3(3 * (m + 2));
  kb.graph_launches = 0;
  bool use_graphs = kb.graphs && kb.graph_key != 0 && !kb.samples;
  if (use_graphs && !arnoldi_graphs_ready(*kb.graphs, kb.graph_key, m)) use_graphs = false;
  GCK(cudaMemcpyAsync(kb.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  double beta = bnorm;
  int total = 0;
  std::vector<double> cycle_beta{bnorm};
  // FP32 basis: v_j is widened into vt for the operators, w = A M^-1 v_j is
  // formed in kb.w (FP64) and stored rounded into the basis once normalised
  const bool f32 = kb.V32 != nullptr && kb.vt != nullptr;
  while (true) {
    if (f32) {
      scale_to_f32_kernel<<<grid_for(n), 256, 0, s>>>(n, 1.0 / beta, kb.r, kb.V32);
      GCK(cudaGetLastError());
    } else {
      // v_0 = r / beta, written without reading the basis (a fresh
      // allocation may hold NaN bit patterns, and 0 * NaN is NaN)
      GCK(la_scale(n, 1.0 / beta, kb.r, kb.V, s));
    }
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    double resid = beta;
    // replayed steps run one ahead: step j + 1 (whose inputs the device
    // forms: v_j+1 is normalised inside step j's graph) is launched before
    // the host waits for step j, so the host's rotations overlap it; a step
    // launched past convergence only writes scratch the solve overwrites
    bool ahead = false;
    for (; j < m && total < maxit; ++j) {
      double* vj = f32 ? kb.vt : kb.V + (size_t)j * n;
      double* vj1 = f32 ? kb.w : kb.V + (size_t)(j + 1) * n;
      const float* vj32 = f32 ? kb.V32 + (size_t)j * n : nullptr;
      float* vj1_32 = f32 ? kb.V32 + (size_t)(j + 1) * n : nullptr;
      if (kb.samples && kb.sample_every > 0 && kb.sample_count < kb.sample_cap && j > 0 &&
          total % kb.sample_every == 0) {
        double* dst = kb.samples + (size_t)kb.sample_count++ * n;
        if (f32) GCK(la_f2d(n, vj32, dst, s));
        else GCK(cudaMemcpyAsync(dst, vj, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      }
      // the step: preconditioner and operator, classical Gram-Schmidt twice
      // (once with cgs_passes = 1) and the norm of the result; the
      // reductions land in separate device slots [pass 1 | pass 2 | |v|^2]
      // and come back in one copy
      auto step = [&](cudaStream_t st, double* host_dst) -> cudaError_t {
        cudaError_t e = f32 ? la_f2d(n, vj32, vj, st) : cudaSuccess;
        if (e == cudaSuccess && M) e = (*M)(vj, kb.z, st);
        if (e == cudaSuccess) e = A(M ? kb.z : vj, vj1, st);
        const int passes = kb.cgs_passes == 1 ? 1 : 2;
        for (int pass = 0; pass < passes && e == cudaSuccess; ++pass) {
          double* slot = kb.dh + (size_t)pass * (m + 2);
          e = f32 ? la_mdot32(*kb.lw, n, kb.V32, n, j + 1, vj1, slot, st)
                  : la_mdot(*kb.lw, n, kb.V, n, j + 1, vj1, slot, st);
          if (e == cudaSuccess)
            e = f32 ? la_maxpy32(n, kb.V32, n, j + 1, slot, -1.0, vj1, st)
                    : la_maxpy(n, kb.V, n, j + 1, slot, -1.0, vj1, st);
        }
        if (e == cudaSuccess) e = la_mdot(*kb.lw, n, vj1, 0, 1, vj1, kb.dh + 2 * (m + 2), st);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(host_dst, kb.dh, sizeof(double) * 3 * (m + 2), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && f32) {
          normalize_to_f32_kernel<<<grid_for(n), 256, 0, st>>>(n, kb.dh + 2 * (m + 2), vj1, vj1_32);
          e = cudaGetLastError();
        }
        return e;
      };
      // replayed from a CUDA graph (which also normalises v_j+1 on the
      // device), or launched one by one
      cudaGraphExec_t gx =
          use_graphs ? arnoldi_graph(*kb.graphs, j, n, vj1, kb.dh + 2 * (m + 2), step, !f32) : nullptr;
      if (gx) {
        ArnoldiGraphs& ag = *kb.graphs;
        if (!ahead) {
          GCK(cudaGraphLaunch(gx, s));
          GCK(cudaEventRecord(ag.done[j & 1], s));
          ++kb.graph_launches;
        }
        ahead = false;
        if (j + 1 < m && total + 1 < maxit && ag.exec[j + 1]) {
          GCK(cudaGraphLaunch(ag.exec[j + 1], s));
          GCK(cudaEventRecord(ag.done[(j + 1) & 1], s));
          ++kb.graph_launches;
          ahead = true;
        }
        GCK(cudaEventSynchronize(ag.done[j & 1]));
        const double* hj = ag.hp + (size_t)(j & 1) * 3 * (m + 2);
        std::copy(hj, hj + 3 * (m + 2), hp3.begin());
      } else {
        GCK(step(s, hp3.data()));
        GCK(cudaStreamSynchronize(s));
      }
      std::fill(hcol.begin(), hcol.end(), 0.0);
      for (int i = 0; i <= j; ++i) hcol[i] += hp3[i] + (kb.cgs_passes == 1 ? 0.0 : hp3[(m + 2) + i]);
      double hn = std::sqrt(hp3[2 * (m + 2)]);
      hcol[j + 1] = hn;
      if (!std::isfinite(hn)) {
        if (err) *err = "non-finite Krylov vector";
        return ICX_ERR_NONFINITE;
      }
      if (!gx && !f32 && hn > 0.0) GCK(la_axpby(n, 1.0 / hn, vj1, 0.0, vj1, s));
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
    if (f32) GCK(la_maxpy32(n, kb.V32, n, j, kb.dh, 1.0, kb.w, s));
    else GCK(la_maxpy(n, kb.V, n, j, kb.dh, 1.0, kb.w, s));
    if (M) {
      GCK((*M)(kb.w, kb.z, s));
      GCK(la_axpby(n, 1.0, kb.z, 1.0, x, s));
    } else {
      GCK(la_axpby(n, 1.0, kb.w, 1.0, x, s));
    }
    GCK(A(x, kb.w, s));
    GCK(la_xpay(n, b, -1.0, kb.w, kb.r, s));
    if (kb.samples && kb.sample_count < kb.sample_cap)
      GCK(cudaMemcpyAsync(kb.samples + (size_t)kb.sample_count++ * n, kb.r, sizeof(double) * n,
                          cudaMemcpyDeviceToDevice, s));
    beta = la_norm(*kb.lw, n, kb.r, kb.dh, s);
    *relres = beta / bnorm;
    if (beta <= tol || total >= maxit || resid <= tol) break;
    cycle_beta.push_back(beta);
    const int nc = (int)cycle_beta.size() - 1;
    if (kb.stall_cycles > 0 && nc >= kb.stall_cycles && beta > 0.9 * cycle_beta[nc - kb.stall_cycles]) break;
  }
  *iters = total;
  return ICX_OK;
}

}  // namespace icx
