// Host side of the tcgen05 BF16 GEMM (icx_gemm_tc.cuh): tensor maps for the
// TMA operand loads, launch shape, split-K, and the C ABI entry point used by
// the tests.
#include <mutex>
#include <string>

#include "../../include/iceicle_b200.h"
#include "icx_gemm_tc.cuh"
#include "icx_internal.h"

namespace icx {
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

std::mutex g_mu;
EncodeTiledFn g_encode = nullptr;
constexpr int MAX_DEV = 64;
int* g_err[MAX_DEV] = {};

cudaError_t encode_fn(EncodeTiledFn* out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    g_encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  *out = g_encode;
  return cudaSuccess;
}

// one device int per GPU for the kernels' timeout flag (zero while healthy)
cudaError_t err_flag(int** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEV) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_err[dev]) {
    e = cudaMalloc((void**)&g_err[dev], sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g_err[dev], 0, sizeof(int));
    if (e != cudaSuccess) {
      g_err[dev] = nullptr;
      return e;
    }
  }
  *out = g_err[dev];
  return cudaSuccess;
}

// rows x cols BF16 matrix, rows ld elements apart, read in boxes of
// box_rows x 64 with the 128-byte swizzle; out-of-range elements read as zero
cudaError_t make_map(CUtensorMap* m, const void* ptr, int rows, int cols, int ld, int box_rows) {
  EncodeTiledFn enc = nullptr;
  cudaError_t e = encode_fn(&enc);
  if (e != cudaSuccess) return e;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)tc::BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int BN>
cudaError_t launch(const CUtensorMap& ma, const CUtensorMap& mb, const tc::Params& p, int nz, cudaStream_t s) {
  static_assert(tc::Smem<BN>::BYTES <= 232448, "operand ring exceeds the shared memory of one CTA");
  cudaError_t e = cudaFuncSetAttribute(tc::gemm_tc_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       tc::Smem<BN>::BYTES);
  if (e != cudaSuccess) return e;
  dim3 grid((p.N + BN - 1) / BN, (p.M + tc::BM - 1) / tc::BM, nz);
  tc::gemm_tc_kernel<BN><<<grid, tc::THREADS, tc::Smem<BN>::BYTES, s>>>(ma, mb, p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t gemm_tc(int M, int N, int K, const tc::bf16_t* A, int lda, const tc::bf16_t* B, int ldb, const float* bias,
                    bool relu, float* C32, int ldc, tc::bf16_t* C16, int ldc16, bool accumulate, int splits, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
  // TMA: 16-byte aligned bases and row strides; K counted in whole 8-value chunks
  if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
    return cudaErrorInvalidValue;
  if (accumulate && (bias || relu || C16 || !C32)) return cudaErrorInvalidValue;
  if (!accumulate && !C32 && !C16) return cudaErrorInvalidValue;
  if (splits < 1) splits = 1;
  int ks = (K + splits - 1) / splits;
  ks = (ks + tc::BK - 1) / tc::BK * tc::BK;  // every split starts on a 64-value (128-byte) boundary
  const int nz = (K + ks - 1) / ks;
  if (nz > 1 && !accumulate) return cudaErrorInvalidValue;
  const bool wide = N > 128;
  const int bn = wide ? 256 : 128;
  CUtensorMap ma, mb;
  cudaError_t e = make_map(&ma, A, M, K, lda, tc::BM);
  if (e == cudaSuccess) e = make_map(&mb, B, N, K, ldb, bn);
  int* err = nullptr;
  if (e == cudaSuccess) e = err_flag(&err);
  if (e != cudaSuccess) return e;
  tc::Params p{M, N, K, ks, bias, relu ? 1 : 0, C32, ldc, C16, ldc16, accumulate ? 1 : 0, err};
  return wide ? launch<256>(ma, mb, p, nz, s) : launch<128>(ma, mb, p, nz, s);
}

// reads and clears the timeout flag of the current device (1: a tile gave up)
cudaError_t gemm_tc_status(int* flag, cudaStream_t s) {
  int* err = nullptr;
  cudaError_t e = err_flag(&err);
  if (e == cudaSuccess) e = cudaMemcpyAsync(flag, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && *flag) e = cudaMemsetAsync(err, 0, sizeof(int), s);
  return e;
}

}  // namespace icx

extern "C" icx_status icx_gemm_bf16_nt(int M, int N, int K, const void* d_A, int lda, const void* d_B, int ldb,
                                       const float* d_bias, int relu, float* d_C32, int ldc, void* d_C16, int ldc16,
                                       int accumulate, int splits, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = icx::gemm_tc(M, N, K, (const icx::tc::bf16_t*)d_A, lda, (const icx::tc::bf16_t*)d_B, ldb, d_bias, relu != 0,
                               d_C32, ldc, (icx::tc::bf16_t*)d_C16, ldc16, accumulate != 0, splits, s);
  if (e == cudaErrorInvalidValue) return ICX_ERR_INVALID;
  if (e != cudaSuccess) return ICX_ERR_CUDA;
  int flag = 0;
  e = icx::gemm_tc_status(&flag, s);
  if (e != cudaSuccess) return ICX_ERR_CUDA;
  return flag ? ICX_ERR_CUDA : ICX_OK;
}
