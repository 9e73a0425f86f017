// BF16 helper kernels of the learned block preconditioner's MLP (its GEMMs
// run on the tcgen05 tensor cores, icx_gemm_tc.cuh).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace icx {

typedef __nv_bfloat16 bf16;

// out[c][r] = in[r][c] for a rows x cols BF16 matrix, out rows ldo apart (32 x
// 32 tiles through shared memory, padded against bank conflicts)
__global__ void transpose_bf16_kernel(int rows, int cols, const bf16* __restrict__ in, bf16* __restrict__ out,
                                      int ldo) {
  __shared__ bf16 t[32][34];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[i][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[(size_t)c * ldo + r] = t[threadIdx.x][i];
  }
}

}  // namespace icx
