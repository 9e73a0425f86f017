// BF16 GEMM on the sm_100a tensor cores: C[M x N] = A[M x K] . B[N x K]^T,
// both operands K-contiguous (row-major, "NT"), FP32 accumulation in tensor
// memory, with the epilogue options of the learned preconditioner's MLP
// (bias over N, ReLU, FP32 and/or BF16 output, or atomic FP32 accumulation
// for split-K partial products).
//
// One CTA of 128 threads per 128 x BN output tile:
//   * warp 0, one lane: TMA producer. Operand tiles of 64 K-values (128 bytes
//     per row, the 128-byte swizzle span) are loaded by cp.async.bulk.tensor
//     into a STAGES-deep ring, each stage signalled by an mbarrier with
//     transaction bytes. No cluster multicast: the operands are this GPU's
//     own memory and every CTA fetches its own tiles.
//   * warp 1, one lane: issues tcgen05.mma (kind::f16, BF16 inputs, M = 128,
//     N = BN, K = 16 per instruction) from shared-memory descriptors into a
//     128 x BN FP32 accumulator in tensor memory, and releases each stage
//     with tcgen05.commit onto the stage's "empty" mbarrier.
//   * all four warps: epilogue. Warp w reads tensor-memory lanes 32w..32w+31
//     (accumulator rows) with tcgen05.ld and writes the outputs.
// Every mbarrier wait is bounded: on timeout the CTA records an error flag,
// skips its stores, frees its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace icx {
namespace tc {

typedef __nv_bfloat16 bf16_t;

constexpr int BM = 128, BK = 64, STAGES = 4, THREADS = 128;
constexpr long long WAIT_LIMIT = 1ll << 24;  // polls of one mbarrier wait (about a second) before giving up

struct Params {
  int M, N, K;
  int k_split;           // K range of blockIdx.z: [z k_split, min(K, (z + 1) k_split)), a multiple of BK
  const float* bias;     // [N] or null
  int relu;
  float* C32;            // [M][ldc] or null
  int ldc;
  bf16_t* C16;           // [M][ldc16] or null
  int ldc16;
  int accumulate;        // C32 += partial tile (atomic), no bias / ReLU / BF16 output
  int* err;              // set to 1 when a wait timed out
};

template <int BN>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int TILES = STAGES * (A_BYTES + B_BYTES);
  // ring of operand tiles (1024-byte aligned for the 128-byte swizzle), then
  // 2 STAGES + 1 mbarriers and the tensor-memory address slot
  static constexpr int BYTES = 1024 + TILES + (2 * STAGES + 1) * 8 + 16;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

// waits until the phase of parity `par` has completed; false after WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned par) {
  const uint32_t a = smem_u32(b);
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(par)
        : "memory");
    if (done) return true;
    if (i > 64) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major operand tile, rows of 128 bytes
// with the 128-byte swizzle, 8-row groups 1024 bytes apart (stride byte
// offset), descriptor version 1 (sm_100), layout type 2 = SWIZZLE_128B
__device__ __forceinline__ uint64_t kmajor_sw128_desc(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A
// and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in bits
// 17-22, M >> 4 in bits 24-28
template <int BN>
__device__ __forceinline__ uint32_t idesc_bf16_f32() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrives on `bar` once every tcgen05.mma issued so far by this thread has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 consecutive accumulator columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Params g) {
  using S = Smem<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = base;
  uint8_t* sB = base + STAGES * S::A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(base + S::TILES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * g.k_split;
  const int kend = min(g.K, kbeg + g.k_split);
  const int nk = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  int issued = 0;  // producer: stages loaded
  if (warp == 0 && lane == 0 && nk > 0) {
    for (int kt = 0; kt < nk; ++kt) {
      const int s = kt % STAGES;
      if (kt >= STAGES && !mbar_wait(&empty[s], (unsigned)((kt / STAGES) - 1) & 1u)) {
        failed = 1;
        break;
      }
      mbar_expect_tx(&full[s], S::A_BYTES + S::B_BYTES);
      const int k0 = kbeg + kt * BK;
      tma_load_2d(sA + s * S::A_BYTES, &tmA, &full[s], k0, m0);
      tma_load_2d(sB + s * S::B_BYTES, &tmB, &full[s], k0, n0);
      ++issued;
    }
  } else if (warp == 1 && lane == 0) {
    const uint32_t idesc = idesc_bf16_f32<BN>();
    for (int kt = 0; kt < nk; ++kt) {
      const int s = kt % STAGES;
      if (!mbar_wait(&full[s], (unsigned)(kt / STAGES) & 1u)) {
        failed = 1;
        break;
      }
      tc_fence_after();
      const uint64_t ad = kmajor_sw128_desc(sA + s * S::A_BYTES), bd = kmajor_sw128_desc(sB + s * S::B_BYTES);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk)  // K step of 16 BF16 = 32 bytes = 2 in the address field
        umma_bf16(tmem, ad + 2ull * kk, bd + 2ull * kk, idesc, (kt | kk) != 0 ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  // epilogue: every warp waits for the accumulator, then reads its 32 lanes
  bool ok = nk > 0 && mbar_wait(done, 0);
  __syncwarp();
  tc_fence_after();
  ok = __all_sync(0xffffffffu, ok ? 1 : 0) != 0;
  if (!ok && nk > 0 && lane == 0) failed = 1;
  __syncthreads();
  if (failed) {
    if (threadIdx.x == 0) atomicExch(g.err, 1);
    // loads already issued complete on their stage barriers before the tiles go away
    if (warp == 0 && lane == 0)
      for (int kt = issued > STAGES ? issued - STAGES : 0; kt < issued; ++kt)
        mbar_wait(&full[kt % STAGES], (unsigned)(kt / STAGES) & 1u);
  } else if (nk > 0) {
    // tcgen05.ld gives lane l the 32 columns of accumulator row 32w + l; a
    // 32 x 33 staging tile in the (now idle) operand ring turns them around
    // so that every store of the warp covers 32 consecutive columns of one
    // output row (one 128-byte line) instead of one word in each of 32 rows
    float* stage = reinterpret_cast<float*>(sA) + warp * 32 * 33;
    const int rbase = m0 + warp * 32;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      if (n0 + c >= g.N) break;  // uniform over the CTA
      float v[32];
      tmem_ld32(lane_addr + (uint32_t)c, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) stage[lane * 33 + j] = v[j];
      __syncwarp();
      const int col = n0 + c + lane;
      const float bcol = (g.bias && col < g.N && !g.accumulate) ? g.bias[col] : 0.f;
#pragma unroll 4
      for (int r = 0; r < 32; ++r) {
        const int row = rbase + r;
        if (row >= g.M || col >= g.N) continue;
        float x = stage[r * 33 + lane];
        if (g.accumulate) {
          atomicAdd(g.C32 + (size_t)row * g.ldc + col, x);
          continue;
        }
        if (g.bias) x += bcol;
        if (g.relu) x = fmaxf(x, 0.f);
        if (g.C32) g.C32[(size_t)row * g.ldc + col] = x;
        if (g.C16) g.C16[(size_t)row * g.ldc16 + col] = __float2bfloat16_rn(x);
      }
      __syncwarp();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
  }
}

}  // namespace tc

// C = A . B^T on the tensor cores (icx_gemm_tc.cu). K, lda, ldb multiples of
// 8, lda and ldb >= K, A and B 16-byte aligned; with splits > 1 only the
// accumulating form (C32 += A . B^T) is allowed.
cudaError_t gemm_tc(int M, int N, int K, const tc::bf16_t* A, int lda, const tc::bf16_t* B, int ldb,
                    const float* bias, bool relu, float* C32, int ldc, tc::bf16_t* C16, int ldc16, bool accumulate,
                    int splits, cudaStream_t s);
// reads (and clears) the flag the GEMM tiles set when a wait timed out
cudaError_t gemm_tc_status(int* flag, cudaStream_t s);
}  // namespace icx
