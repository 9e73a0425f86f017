// Block-ILU(0) apply pipelined by grid rows, for the natural element order of
// one nx x ny structured grid (element e = i + nx j; its strictly lower
// neighbours are e - nx and e - 1, its strictly upper ones e + 1 and e + nx):
//
//   forward   f_e = x_e - L_{e,e-nx} f_{e-nx} - L_{e,e-1} f_{e-1}        i = 0 .. nx-1
//   backward  y_e = inv(U_ee) f_e - (inv(U_ee) U)_{e,e+1} y_{e+1}
//                                 - (inv(U_ee) U)_{e,e+nx} y_{e+nx}   i = nx-1 .. 0
//
// One CTA owns grid row j and runs its elements in order, first the forward
// sweep, then the backward sweep. The dependency along the row stays inside
// the CTA (the previous element's result is kept in shared memory), so only
// the dependency on the neighbouring row crosses CTAs: element (i, j) of the
// forward sweep waits for the completion counter of (i, j-1), of the backward
// sweep for that of (i, j+1). Rows therefore run as a wavefront skewed by one
// element, and the critical path is nx + ny element steps of which only ny
// wait on another CTA (the data-flow apply waits at every one of its nx + ny
// levels). While one element is computed, the matrix blocks of the next are
// already on their way into shared memory (cp.async, two stages where they
// fit).
//
// Every product reads its block as consecutive VEC-element vectors (thread t
// takes vectors t, t + THREADS, ...), accumulates the partial sums of its
// fixed (row, column group) positions over the element's blocks, and the row
// sums are formed from those partials in a fixed order, so the result does not
// depend on scheduling.
//
// Waits: thread 0 polls the counter with acquire loads, bounded by
// ICX_FLOW_SPINS polls and abandoned when *err is set; a timeout sets *err = 1,
// an index that does not fit the grid pattern *err = 2. The rows are all
// resident (cooperative launch of ny CTAs, checked against the occupancy), so
// every wait ends: each dependency is an earlier element of a row that never
// waits on a later row in the same sweep.
#pragma once
#include <cuda_runtime.h>

#include "icx_blockrow.cuh"

namespace icx {

template <class TA>
struct IluRowArgs {
  int nx, ny, nnzb;
  const int* rowptr;
  const int* colidx;
  const int* diag;
  const TA* LU;    // strictly lower blocks L, upper blocks inv(U_ee) U_ek
  const TA* Uinv;  // [E] inv(U_ee)
  const double* x;
  double* f;       // forward result
  double* y;       // output
  unsigned* cnt_f;
  unsigned* cnt_b;
  unsigned epoch;
  int* err;
};

template <int BS, class TA>
struct IluRowCfg {
  static constexpr int THREADS = 128;
  static constexpr int VEC = (sizeof(TA) == 4 && BS % 4 == 0) ? 4 : (BS % 2 == 0 ? 2 : 1);
  static constexpr int QR = BS / VEC;                   // vectors per block row
  static constexpr int Q = BS * QR;                     // vectors per block
  static constexpr int J = (Q + THREADS - 1) / THREADS; // vectors per thread and block
  static constexpr int MAXB = 3;                        // blocks per element and sweep
  static constexpr int STAGE = MAXB * BS * BS;          // TA per prefetch stage
  static constexpr int STAGES = (2 * STAGE * sizeof(TA) <= 200 * 1024) ? 2 : 1;
  static constexpr size_t TA_BYTES = (sizeof(TA) * (STAGES * STAGE + Q + MAXB * BS) + 15) / 16 * 16;
  static constexpr size_t SMEM = TA_BYTES + sizeof(double) * BS + 16;
};

__device__ inline void cp_async_4(void* sdst, const void* gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ inline void cp_async_8(void* sdst, const void* gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ inline void cp_async_16(void* sdst, const void* gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
// cp_async_commit / cp_async_wait<N>: icx_blockrow.cuh

// copy `count` TA values (a multiple of 16 bytes when `vec16`) from global to shared
template <class TA>
__device__ inline void copy_async(TA* sdst, const TA* gsrc, int count, bool vec16) {
  if (vec16) {
    constexpr int PER = 16 / sizeof(TA);
    for (int k = threadIdx.x * PER; k < count; k += blockDim.x * PER) cp_async_16(sdst + k, gsrc + k);
  } else {
    for (int k = threadIdx.x; k < count; k += blockDim.x) {
      if (sizeof(TA) == 8) cp_async_8(sdst + k, gsrc + k);
      else cp_async_4(sdst + k, gsrc + k);
    }
  }
}

// thread 0 waits (bounded) for *c to reach target; the CTA learns the outcome
__device__ inline bool row_wait(const unsigned* c, unsigned target, int* err, int* s_flag) {
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned spins = 0;
    while ((int)(ld_acquire_u32(c) - target) < 0) {
      if (*reinterpret_cast<volatile int*>(err)) { ok = 0; break; }
      if (++spins > ICX_FLOW_SPINS) { atomicExch(err, 1); ok = 0; break; }
    }
    *s_flag = ok;
  }
  __syncthreads();
  return *reinterpret_cast<volatile int*>(s_flag) != 0;
}

// the CTA's stores of this element are ordered before thread 0's release by
// the barrier (causality through the CTA-scope barrier and the gpu-scope
// release / acquire pair, as the warp-level signal of the data-flow apply)
__device__ inline void row_signal(unsigned* c) {
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(c) : "memory");
}

template <int BS, class TA>
__global__ void __launch_bounds__(128) ilu_apply_rows_kernel(IluRowArgs<TA> a) {
  using K = IluRowCfg<BS, TA>;
  constexpr int VEC = K::VEC, QR = K::QR, Q = K::Q, J = K::J, D = BS * BS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TA* s_blk = reinterpret_cast<TA*>(smem_raw);           // [STAGES][MAXB][BS*BS]
  TA* s_part = s_blk + K::STAGES * K::STAGE;            // [Q]
  TA* s_v = s_part + Q;                                 // [MAXB][BS] vectors the blocks multiply
  double* s_prev = reinterpret_cast<double*>(smem_raw + K::TA_BYTES);  // [BS] previous element's result
  int* s_flag = reinterpret_cast<int*>(s_prev + BS);
  const int j = blockIdx.x, nx = a.nx, E = a.nx * a.ny;
  const int t = threadIdx.x;
  const bool vec16 = (D * sizeof(TA)) % 16 == 0;
  if (j >= a.ny) return;

  // block positions of element e for a sweep: the expected neighbours in
  // order, checked against the pattern (uniform over the CTA)
  // own[b]: the block's neighbour is the previous element of this row (its
  // result is in s_prev), not one of the neighbouring row (even when the two
  // have the same index, as for nx = 1)
  auto blocks_of = [&](int e, bool fwd, int* kb, int* col, bool* own) -> int {
    const int i = e - nx * (e / nx), jj = e / nx;
    const int d = a.diag[e], rb = a.rowptr[e], re = a.rowptr[e + 1];
    int n = 0;
    if (fwd) {
      if (jj > 0) { kb[n] = rb + n; col[n] = e - nx; own[n] = false; ++n; }
      if (i > 0) { kb[n] = rb + n; col[n] = e - 1; own[n] = true; ++n; }
      if (rb + n != d) return -1;
    } else {
      if (i < nx - 1) { kb[n] = d + 1 + n; col[n] = e + 1; own[n] = true; ++n; }
      if (jj < a.ny - 1) { kb[n] = d + 1 + n; col[n] = e + nx; own[n] = false; ++n; }
      if (d + 1 + n != re) return -1;
    }
    for (int b = 0; b < n; ++b)
      if (kb[b] < 0 || kb[b] >= a.nnzb || a.colidx[kb[b]] != col[b]) return -1;
    return n;
  };
  // start the copies of element e's blocks into stage st
  auto prefetch = [&](int e, bool fwd, int st) -> int {
    int kb[2], col[2];
    bool own[2];
    const int n = blocks_of(e, fwd, kb, col, own);
    if (n < 0) return -1;
    TA* dst = s_blk + st * K::STAGE;
    if (n > 0) copy_async(dst, a.LU + (size_t)kb[0] * D, n * D, vec16);  // the element's neighbour blocks are adjacent
    if (!fwd) copy_async(dst + n * D, a.Uinv + (size_t)e * D, D, vec16);
    cp_async_commit();
    return n;
  };

  for (int sweep = 0; sweep < 2; ++sweep) {
    const bool fwd = sweep == 0;
    const unsigned* wait_cnt = fwd ? a.cnt_f : a.cnt_b;
    unsigned* sig_cnt = fwd ? a.cnt_f : a.cnt_b;
    const int e0 = fwd ? nx * j : nx * j + nx - 1;
    const int step = fwd ? 1 : -1;
    int n_cur = prefetch(e0, fwd, 0);
    for (int ii = 0; ii < nx; ++ii) {
      const int e = e0 + step * ii, st = K::STAGES == 2 ? (ii & 1) : 0;
      if (n_cur < 0) {
        if (t == 0) atomicExch(a.err, 2);
        cp_async_wait<0>();
        return;
      }
      int n_next = 0;
      const bool more = ii + 1 < nx;
      if (K::STAGES == 2 && more) n_next = prefetch(e + step, fwd, st ^ 1);
      // the neighbouring row's element (the copies of this element's blocks overlap the wait)
      const int other = fwd ? e - nx : e + nx;
      if (other >= 0 && other < E)
        if (!row_wait(wait_cnt + other, a.epoch, a.err, s_flag)) {
          cp_async_wait<0>();
          return;
        }
      if (K::STAGES == 2 && more) cp_async_wait<1>();
      else cp_async_wait<0>();
      // vectors in the block order of blocks_of (backward: then f_e for inv(U_ee))
      {
        int kb[2], col[2];
        bool own[2];
        const int n = blocks_of(e, fwd, kb, col, own);
        for (int c = t; c < BS; c += K::THREADS) {
          for (int b = 0; b < n; ++b)
            s_v[b * BS + c] = (TA)(own[b] ? s_prev[c] : __ldcg((fwd ? a.f : a.y) + (size_t)col[b] * BS + c));
          if (!fwd) s_v[n * BS + c] = (TA)__ldcg(a.f + (size_t)e * BS + c);
        }
      }
      __syncthreads();
      const int nb = fwd ? n_cur : n_cur + 1;
      const TA* blk = s_blk + st * K::STAGE;
      TA acc[J];
#pragma unroll
      for (int jj = 0; jj < J; ++jj) acc[jj] = TA(0);
      for (int b = 0; b < nb; ++b) {
        // forward: every block is subtracted; backward: inv(U_ee) (last) added, the others subtracted
        const TA sg = (!fwd && b == nb - 1) ? TA(1) : TA(-1);
#pragma unroll
        for (int jj = 0; jj < J; ++jj) {
          const int q = t + jj * K::THREADS;
          if (q < Q) {
            const TA* p = blk + (size_t)b * D + (size_t)q * VEC;
            const int c0 = (q % QR) * VEC;
            TA s = TA(0);
#pragma unroll
            for (int v = 0; v < VEC; ++v) s += p[v] * s_v[b * BS + c0 + v];
            acc[jj] += sg * s;
          }
        }
      }
#pragma unroll
      for (int jj = 0; jj < J; ++jj) {
        const int q = t + jj * K::THREADS;
        if (q < Q) s_part[q] = acc[jj];
      }
      __syncthreads();
      for (int r = t; r < BS; r += K::THREADS) {
        TA sum = TA(0);
#pragma unroll
        for (int g = 0; g < QR; ++g) sum += s_part[r * QR + g];
        const double v = fwd ? a.x[(size_t)e * BS + r] + (double)sum : (double)sum;
        s_prev[r] = v;
        __stcg((fwd ? a.f : a.y) + (size_t)e * BS + r, v);
      }
      row_signal(sig_cnt + e);
      if (K::STAGES == 1 && more) n_next = prefetch(e + step, fwd, 0);
      n_cur = n_next;
    }
    __syncthreads();
  }
}

}  // namespace icx
