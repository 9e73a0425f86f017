// In-place Gauss-Jordan inversion of a small dense block in shared memory by
// one CTA, shared by the block-Jacobi and block-ILU(0) preconditioners and the
// element mass-matrix inverses of the explicit time steppers.
#pragma once
#include <cuda_runtime.h>

namespace icx {

// In-place Gauss-Jordan inversion with partial pivoting of the BS x BS block
// `a` in shared memory by the whole CTA (blockDim.x >= 2 BS), three barriers
// per pivot step:
//   1. warp 0 finds the pivot row p of column k (largest |a[i][k]|, i >= k,
//      first index on ties) and keeps a[p][k] and a[k][k];
//   2. column threads swap rows k and p and scale row k by 1/pivot (a[k][k]
//      becomes 1/pivot); row threads save the multipliers f_i = a[i][k];
//   3. every entry off row k: a[i][j] -= f_i a[k][j] (j != k), a[i][k] = -f_i a[k][k].
// The row interchanges are undone as a column permutation when the result is
// written out (write_inverse). A zero pivot sets *singular and stops.
template <int BS>
__device__ void gj_invert(double* a, int* perm, double* fcol, int* singular) {
  __shared__ int s_p;
  __shared__ double s_pv, s_akk;
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) *singular = 0;
  __syncthreads();
  for (int k = 0; k < BS; ++k) {
    if (tid < 32) {
      double best = -1.0;
      int bi = BS;
      for (int i = k + lane; i < BS; i += 32) {
        double v = fabs(a[i * BS + k]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, best, off);
        int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
      }
      if (lane == 0) {
        s_p = bi;
        perm[k] = bi;
        s_pv = a[bi * BS + k];
        s_akk = a[k * BS + k];
        if (!(best > 0.0)) *singular = 1;
      }
    }
    __syncthreads();
    if (*singular) return;
    const int p = s_p;
    const double pv = s_pv;
    if (tid < BS) {
      const int j = tid;
      double rk = a[k * BS + j], rp = a[p * BS + j];
      if (p != k) a[p * BS + j] = rk;
      a[k * BS + j] = (j == k ? 1.0 : rp) / pv;
    } else if (tid >= 128 && tid < 128 + BS) {
      const int i = tid - 128;
      fcol[i] = (i == p) ? s_akk : a[i * BS + k];
    }
    __syncthreads();
    const double akk = a[k * BS + k];
    for (int t = tid; t < BS * BS; t += blockDim.x) {
      int i = t / BS, j = t - i * BS;
      if (i == k) continue;
      if (j == k) a[t] = -fcol[i] * akk;
      else a[t] -= fcol[i] * a[k * BS + j];
    }
    __syncthreads();
  }
}

// dst = the inverse held in `a` after gj_invert, with the row interchanges
// undone as column interchanges in reverse order (composed into one gather);
// the identity if the block was singular
template <int BS>
__device__ void write_inverse(const double* a, const int* perm, int* colsrc, int singular, double* dst) {
  if (threadIdx.x == 0 && !singular) {
    for (int j = 0; j < BS; ++j) colsrc[j] = j;
    for (int k = BS - 1; k >= 0; --k) {
      int p = perm[k];
      if (p != k) { int t = colsrc[k]; colsrc[k] = colsrc[p]; colsrc[p] = t; }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < BS * BS; t += blockDim.x) {
    int i = t / BS, j = t - i * BS;
    dst[t] = singular ? (i == j ? 1.0 : 0.0) : a[i * BS + colsrc[j]];
  }
}

template <int BS>
struct InvSmem {
  static constexpr size_t BYTES = sizeof(double) * (BS * BS + BS) + sizeof(int) * 2 * BS;
};

}  // namespace icx
