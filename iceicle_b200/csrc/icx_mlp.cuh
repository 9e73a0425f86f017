// BF16 kernels of the learned block preconditioner's MLP: a tensor-core GEMM
// (mma.sync m16n8k16, BF16 operands, FP32 accumulation) and the elementwise,
// transpose and reduction kernels of its forward and backward passes.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace icx {

typedef __nv_bfloat16 bf16;

// C[M x N] = A[M x K] . B[N x K]^T (both operands K-contiguous, row-major),
// with an optional bias over N and ReLU, written as FP32 and/or BF16; or
// (accumulate) added atomically into C32, which is how split-K (blockIdx.z
// takes K range [z * k_split, (z + 1) * k_split)) combines its partial tiles.
// Requirements checked by the launcher: K, lda, ldb multiples of 8 and A, B
// 16-byte aligned (every staged chunk is 8 BF16 values, 16 bytes).
struct GemmArgs {
  int M, N, K;
  const bf16* A;
  int lda;
  const bf16* B;
  int ldb;
  const float* bias;
  int relu;
  float* C32;
  int ldc;
  bf16* C16;
  int ldc16;
  int accumulate;
  int k_split;
};

constexpr int GEMM_BM = 128, GEMM_BN = 128, GEMM_BK = 32, GEMM_PAD = 8;

__device__ inline void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// 256 threads: 2 x 4 warps, each 64 (M) x 32 (N) of the 128 x 128 tile. Shared
// rows are padded to 40 BF16 (20 words): the fragment reads of a warp (rows
// g = lane / 4, word t = lane % 4) then hit 32 distinct banks.
__global__ void __launch_bounds__(256) gemm_bf16_nt_kernel(GemmArgs g) {
  __shared__ __align__(16) bf16 As[GEMM_BM][GEMM_BK + GEMM_PAD];
  __shared__ __align__(16) bf16 Bs[GEMM_BN][GEMM_BK + GEMM_PAD];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;
  const int m0 = blockIdx.y * GEMM_BM, n0 = blockIdx.x * GEMM_BN;
  const int kbeg = blockIdx.z * g.k_split;
  const int kend = min(g.K, kbeg + g.k_split);
  const int grp = lane >> 2, tq = lane & 3;
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.f;
  constexpr int CH = GEMM_BK / 8;  // 16-byte chunks per tile row
  for (int k0 = kbeg; k0 < kend; k0 += GEMM_BK) {
    for (int c = tid; c < GEMM_BM * CH; c += 256) {
      const int r = c / CH, kc = (c % CH) * 8;
      const int gr = m0 + r, gk = k0 + kc;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gr < g.M && gk < kend) v = *reinterpret_cast<const uint4*>(g.A + (size_t)gr * g.lda + gk);
      *reinterpret_cast<uint4*>(&As[r][kc]) = v;
    }
    for (int c = tid; c < GEMM_BN * CH; c += 256) {
      const int r = c / CH, kc = (c % CH) * 8;
      const int gn = n0 + r, gk = k0 + kc;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gn < g.N && gk < kend) v = *reinterpret_cast<const uint4*>(g.B + (size_t)gn * g.ldb + gk);
      *reinterpret_cast<uint4*>(&Bs[r][kc]) = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GEMM_BK; kk += 16) {
      uint32_t af[4][4], bfr[4][2];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const int r = wm + mi * 16 + grp;
        af[mi][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tq]);
        af[mi][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tq]);
        af[mi][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tq + 8]);
        af[mi][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tq + 8]);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int n = wn + ni * 8 + grp;
        bfr[ni][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * tq]);
        bfr[ni][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * tq + 8]);
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_bf16_16816(acc[mi][ni], af[mi], bfr[ni]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int r = m0 + wm + mi * 16 + grp + (v >= 2 ? 8 : 0);
        const int col = n0 + wn + ni * 8 + 2 * tq + (v & 1);
        if (r >= g.M || col >= g.N) continue;
        float x = acc[mi][ni][v];
        if (g.accumulate) {
          atomicAdd(g.C32 + (size_t)r * g.ldc + col, x);
          continue;
        }
        if (g.bias) x += g.bias[col];
        if (g.relu) x = fmaxf(x, 0.f);
        if (g.C32) g.C32[(size_t)r * g.ldc + col] = x;
        if (g.C16) g.C16[(size_t)r * g.ldc16 + col] = __float2bfloat16_rn(x);
      }
}

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
