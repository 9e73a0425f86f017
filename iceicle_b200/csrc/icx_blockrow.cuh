// Block-row products on the element block pattern, shared by the BSR SpMV,
// the block-diagonal apply and the block-ILU(0) triangular solves:
//
//   y_e[r] = x0_e[r] + sign * sum_{blocks (e, k) selected} A_ek[r][:] . v_k
//
// One warp computes R consecutive rows of one block row. Lane l holds columns
// l, l + 32, ... of every row it touches, so each load of a block row is one
// contiguous 256-byte segment; the R partial sums are reduced across the warp
// with butterfly shuffles and lane rr stores row r0 + rr.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <type_traits>

namespace icx {

enum BlockRowMode {
  BR_ALL = 0,    // every block of the row (SpMV)
  BR_LOWER = 1,  // the blocks left of the diagonal (column < row)
  BR_UPPER = 2,  // the blocks right of the diagonal (column > row)
  BR_DIAG = 3    // block-diagonal storage D[e] (one block per row, column = row)
};

// a * b + c rounded once: the ILU applies state every product-sum as an
// explicit fused multiply-add, so their variants round alike whatever the
// compiler would contract
__device__ inline float fused_madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ inline double fused_madd(double a, double b, double c) { return __fma_rn(a, b, c); }

// Warp sums of R per-lane partial rows by a butterfly reduce-scatter: at
// distance 16, 8, ... each lane keeps half of its rows, adding its partner's
// copy of them, until one row is left, then finishes with the plain
// butterfly. Every addition is one the full butterfly (acc += shfl_xor(acc,
// d), d = 16 .. 1, on every row) also makes, so each row's sum is the same
// value, with about R + 5 shuffles instead of 5 R. Lane l ends with the sum
// of row `row` (from its bits 4, 3, ...); `owner` marks one lane per row
// below R.
template <class T>
struct RowSum {
  T v;
  int row;
  bool owner;
};

template <int R, class T>
__device__ inline RowSum<T> warp_row_sums(const T (&acc)[R]) {
  static_assert(R >= 1 && R <= 32, "rows per warp task");
  constexpr int RP = R <= 1 ? 1 : R <= 2 ? 2 : R <= 4 ? 4 : R <= 8 ? 8 : R <= 16 ? 16 : 32;
  const int lane = threadIdx.x & 31;
  T v[RP];
#pragma unroll
  for (int i = 0; i < RP; ++i) v[i] = i < R ? acc[i] : T(0);
  int row = 0, d = 16;
#pragma unroll
  for (int m = RP; m > 1; m >>= 1, d >>= 1) {
    const bool hi = (lane & d) != 0;
#pragma unroll
    for (int i = 0; i < m / 2; ++i) {
      const T send = hi ? v[i] : v[i + m / 2];
      const T keep = hi ? v[i + m / 2] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, d);
    }
    if (hi) row += m / 2;
  }
#pragma unroll
  for (; d > 0; d >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], d);
  return {v[0], row, row < R && (lane & (32 / RP - 1)) == 0};
}

// the block rows 0..nrows-1 of one launch
struct RowSet {
  int nx, ny, level, nrows;
  __host__ __device__ int count() const { return nrows; }
  __device__ int row(int idx) const { return idx; }
};

template <int BS>
struct BlockRowCfg {
  static constexpr int NS = (BS + 31) / 32;                   // column chunks per lane
  static constexpr int R = BS >= 64 ? 8 : (BS >= 32 ? 4 : 2);  // rows per warp
  static constexpr int GROUPS = (BS + R - 1) / R;             // warps per block row
};

template <int BS, int MODE, bool COHERENT, class TA = double>
__device__ inline void block_row_task(const RowSet& rs, long long task, const int* __restrict__ rowptr,
                                      const int* __restrict__ colidx, const TA* __restrict__ A,
                                      const double* v, const double* x0, double sign, double* y) {
  using K = BlockRowCfg<BS>;
  constexpr int NS = K::NS, R = K::R;
  const int lane = threadIdx.x & 31;
  const int idx = (int)(task / K::GROUPS), g = (int)(task - (long long)idx * K::GROUPS);
  const int e = rs.row(idx);
  const int r0 = g * R;
  TA acc[R];
#pragma unroll
  for (int rr = 0; rr < R; ++rr) acc[rr] = TA(0);
  int kb0, kb1;
  if (MODE == BR_DIAG) { kb0 = e; kb1 = e + 1; }
  else { kb0 = rowptr[e]; kb1 = rowptr[e + 1]; }
  for (int kb = kb0; kb < kb1; ++kb) {
    const int k = MODE == BR_DIAG ? e : colidx[kb];
    if ((MODE == BR_LOWER && k >= e) || (MODE == BR_UPPER && k <= e)) continue;
    TA xv[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      int c = lane + 32 * s;
      xv[s] = c < BS ? (TA)(COHERENT ? __ldcg(v + (size_t)k * BS + c) : v[(size_t)k * BS + c]) : TA(0);
    }
    const TA* Ab = A + (size_t)kb * BS * BS;
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      int r = r0 + rr;
      if (r < BS) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          int c = lane + 32 * s;
          if (c < BS) acc[rr] += Ab[(size_t)r * BS + c] * xv[s];
        }
      }
    }
  }
  const RowSum<TA> sum = warp_row_sums<R>(acc);
  const TA mine = sum.v;
  const int r = r0 + sum.row;
  if (sum.owner && r < BS) {
    double base = x0 ? (COHERENT ? __ldcg(x0 + (size_t)e * BS + r) : x0[(size_t)e * BS + r]) : 0.0;
    y[(size_t)e * BS + r] = base + sign * (double)mine;
  }
}

template <int BS, int MODE, class TA = double>
__global__ void __launch_bounds__(256) block_row_kernel(RowSet rs, const int* __restrict__ rowptr,
                                                        const int* __restrict__ colidx,
                                                        const TA* __restrict__ A, const double* v,
                                                        const double* x0, double sign, double* y) {
  const long long task = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (task >= (long long)rs.count() * BlockRowCfg<BS>::GROUPS) return;
  block_row_task<BS, MODE, false, TA>(rs, task, rowptr, colidx, A, v, x0, sign, y);
}

// Small blocks (BS <= 36): one warp per block row, reading each block as one
// contiguous run of VEC-element vectors (16 bytes where BS allows): lane l
// takes vectors l, l + 32, ..., so every load instruction of the warp moves a
// contiguous 512-byte segment. A lane's vectors sit at the same (row, column
// group) positions in every block of the row, so its partial sums stay in
// registers across the row's blocks; they are combined once per block row
// through shared memory, row r adding its BS / VEC column groups in a fixed
// order (the result does not depend on scheduling).
template <class TA, int BS>
struct VecRowCfg {
  static constexpr int VEC = (sizeof(TA) == 4 && BS % 4 == 0) ? 4 : (BS % 2 == 0 ? 2 : 1);
  static constexpr int QR = BS / VEC;       // vectors per block row
  static constexpr int Q = BS * QR;         // vectors per block
  static constexpr int J = (Q + 31) / 32;   // vectors per lane
  static constexpr int NCH = (sizeof(TA) == 8 && J > 12) ? 2 : 1;  // load chunks per block
  static constexpr int JC = (J + NCH - 1) / NCH;                   // vectors per lane per chunk
  static constexpr int WARPS = 8;
};

template <class TA, int VEC>
__device__ inline void load_vec(const TA* __restrict__ p, TA (&o)[VEC]) {
  if constexpr (sizeof(TA) == 4 && VEC == 4) {
    float4 t = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
  } else if constexpr (sizeof(TA) == 4 && VEC == 2) {
    float2 t = __ldg(reinterpret_cast<const float2*>(p));
    o[0] = t.x; o[1] = t.y;
  } else if constexpr (sizeof(TA) == 8 && VEC == 2) {
    double2 t = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = t.x; o[1] = t.y;
  } else {
#pragma unroll
    for (int t = 0; t < VEC; ++t) o[t] = __ldg(p + t);
  }
}

// two CTAs (16 warps) per SM at most 128 registers: without the bound the
// 36 x 36 FP64 variant holds a whole block row's loads (170 registers, one CTA)
template <class TA, int BS>
constexpr int vec_row_min_blocks() { return (sizeof(TA) == 8 && BS >= 25) ? 2 : 1; }

template <int BS, int MODE, class TA>
__global__ void __launch_bounds__(256, vec_row_min_blocks<TA, BS>()) block_row_vec_kernel(int nrows, const int* __restrict__ rowptr,
                                                            const int* __restrict__ colidx,
                                                            const TA* __restrict__ A, const double* v,
                                                            const double* x0, double sign, double* y) {
  using K = VecRowCfg<TA, BS>;
  constexpr int VEC = K::VEC, QR = K::QR, Q = K::Q, J = K::J;
  __shared__ TA xs_all[K::WARPS][BS];
  __shared__ TA part_all[K::WARPS][Q];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * K::WARPS + wid;
  if (e >= nrows) return;  // uniform over the warp; only warp-level barriers follow
  TA* xs = xs_all[wid];
  TA* part = part_all[wid];
  TA acc[J];
#pragma unroll
  for (int j = 0; j < J; ++j) acc[j] = TA(0);
  int kb0, kb1;
  if (MODE == BR_DIAG) { kb0 = e; kb1 = e + 1; }
  else { kb0 = rowptr[e]; kb1 = rowptr[e + 1]; }
  for (int kb = kb0; kb < kb1; ++kb) {
    const int k = MODE == BR_DIAG ? e : colidx[kb];
    if ((MODE == BR_LOWER && k >= e) || (MODE == BR_UPPER && k <= e)) continue;
    const TA* Ab = A + (size_t)kb * BS * BS;
    // the block's vectors in NCH chunks of JC per lane (one chunk for FP32;
    // two for large FP64 blocks, which keeps them within 128 registers); the
    // first chunk's loads are in flight while x_k is staged
#pragma unroll
    for (int ch = 0; ch < K::NCH; ++ch) {
      TA a[K::JC][VEC];
#pragma unroll
      for (int jj = 0; jj < K::JC; ++jj) {
        const int j = ch * K::JC + jj, q = lane + 32 * j;
        if (j < J && q < Q) load_vec<TA, VEC>(Ab + (size_t)q * VEC, a[jj]);
        else {
#pragma unroll
          for (int t = 0; t < VEC; ++t) a[jj][t] = TA(0);
        }
      }
      if (ch == 0) {
        for (int c = lane; c < BS; c += 32) xs[c] = (TA)v[(size_t)k * BS + c];
        __syncwarp();
      }
#pragma unroll
      for (int jj = 0; jj < K::JC; ++jj) {
        const int j = ch * K::JC + jj, q = lane + 32 * j;
        if (j < J && q < Q) {
          const int c0 = (q % QR) * VEC;
#pragma unroll
          for (int t = 0; t < VEC; ++t) acc[j] += a[jj][t] * xs[c0 + t];
        }
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int q = lane + 32 * j;
    if (q < Q) part[q] = acc[j];
  }
  __syncwarp();
  for (int r = lane; r < BS; r += 32) {
    TA sum = TA(0);
#pragma unroll
    for (int g = 0; g < QR; ++g) sum += part[r * QR + g];
    const double base = x0 ? x0[(size_t)e * BS + r] : 0.0;
    y[(size_t)e * BS + r] = base + sign * (double)sum;
  }
}

// launch over a row set: 8 warps per CTA
template <int BS, int MODE, class TA = double>
inline cudaError_t launch_block_rows(const RowSet& rs, const int* rowptr, const int* colidx, const TA* A,
                                     const double* v, const double* x0, double sign, double* y, cudaStream_t s) {
  if constexpr (BS <= 36) {
    const int n = rs.count();
    if (n <= 0) return cudaSuccess;
    constexpr int W = VecRowCfg<TA, BS>::WARPS;
    block_row_vec_kernel<BS, MODE, TA><<<(n + W - 1) / W, W * 32, 0, s>>>(n, rowptr, colidx, A, v, x0, sign, y);
    return cudaGetLastError();
  } else {
    long long tasks = (long long)rs.count() * BlockRowCfg<BS>::GROUPS;
    if (tasks <= 0) return cudaSuccess;
    unsigned blocks = (unsigned)((tasks + 7) / 8);
    block_row_kernel<BS, MODE, TA><<<blocks, 256, 0, s>>>(rs, rowptr, colidx, A, v, x0, sign, y);
    return cudaGetLastError();
  }
}


// ---------------------------------------------------------------------------
// Block-ILU(0) apply in one cooperative launch, scheduled by data flow:
//   forward   f_e = x_e - sum_{k<e} L_ek f_k                      (levels ascending)
//   backward  y_e = inv(U_ee) f_e - sum_{k>e} (inv(U_ee) U_ek) y_k  (levels descending)
// A task is (element, group of R rows). The tasks are ordered by level (the
// element order `order` lists the elements by level, the anti-diagonal i + j
// of the element in its grid; every strictly lower neighbour of an element is
// on a lower level) and dealt to the
// warps round-robin; every warp runs its tasks in that order, all forward
// tasks before any backward task. A task loads its matrix rows, then waits
// only for the elements it reads, on one of two schedules:
//   sentinel (the default): the outputs are pre-filled with a sentinel value
//     and the waiting warp polls the values it reads until none holds it
//     (below, FLOW_SENTINEL);
//   counters: each element has a completion counter per sweep that every
//     group increments after writing its rows, and the sweep of apply number
//     `epoch` is complete for element k when its counter reaches
//     epoch * GROUPS (the counters grow across applies; the solver zeroes
//     them when GROUPS changes).
// Because every dependency is a task earlier in some warp's order and all
// warps are resident (cooperative launch), the waits always end; each is
// nevertheless bounded by ICX_FLOW_SPINS polls, after which the warp sets
// *err and the launch winds down (every waiting warp polls *err).
#ifndef ICX_FLOW_SPINS
#define ICX_FLOW_SPINS (1u << 22)
#endif

template <class TA>
struct IluFlowArgs {
  int E, nnzb;
  const int* rowptr;
  const int* colidx;
  const int* diag;      // position of each row's diagonal block
  const int* order;     // [E] elements by ascending level
  const TA* LU;         // strictly lower blocks L, upper blocks inv(U_ee) U_ek
  const TA* Uinv;       // [E] inv(U_ee)
  const double* x;
  double* f;            // forward result
  double* y;            // output
  unsigned* cnt_f;      // [E] forward completion counters
  unsigned* cnt_b;      // [E] backward completion counters
  unsigned epoch;
  int* err;
};

// acquire load of a completion counter: the waiting warp's later loads of the
// producer's data are ordered after the observation (__syncwarp then orders
// them for the other lanes); counters are compared wrap-safe
__device__ inline unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// up to three counters at once: lane k < n polls counter k with acquire loads
// until every one has reached target (warp vote), so the waits overlap. At most
// ICX_FLOW_SPINS polls: then *err = 1; a set *err ends the wait early. Returns
// false in both cases. __syncwarp then orders each lane's acquire before the
// loads of every lane.
__device__ inline bool flow_wait_n(const unsigned* c0, const unsigned* c1, const unsigned* c2, int n,
                                   unsigned target, int* err) {
  const int lane = threadIdx.x & 31;
  const unsigned* c = lane == 0 ? c0 : (lane == 1 ? c1 : c2);
  bool done = lane >= n;
  unsigned spins = 0;
  int ok = 1;
  while (true) {
    if (!done) done = (int)(ld_acquire_u32(c) - target) >= 0;
    if (__all_sync(0xffffffffu, done)) break;
    int stop = 0;
    if (lane == 0) {
      if (*reinterpret_cast<volatile int*>(err)) stop = 1;
      else if (++spins > ICX_FLOW_SPINS) {
        atomicExch(err, 1);
        stop = 1;
      }
    }
    if (__shfl_sync(0xffffffffu, stop, 0)) {
      ok = 0;
      break;
    }
  }
  __syncwarp();
  return ok != 0;
}

// the warp's stores happen before the increment (release at gpu scope,
// cumulative over the lanes' stores ordered by __syncwarp)
__device__ inline void flow_signal(unsigned* c) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(c) : "memory");
}

// Sentinel schedule of the same apply: instead of counting completed tasks,
// every output slot (f and y) is filled with FLOW_SENTINEL before the launch,
// each task stores its rows with relaxed stores (no fence, no counter), and a
// waiting warp loads the values it reads with relaxed loads until none holds
// the sentinel. Each 8-byte value is observed whole, so no ordering between a
// task's stores is needed: a level costs one store and one polled load
// instead of a fence, a counter update, a counter poll and a load. The
// sentinel is a NaN whose payload FP64 arithmetic never returns (results that
// are NaN carry the canonical payload), and the outputs are always results
// of arithmetic.
constexpr unsigned long long FLOW_SENTINEL = 0x7FF4B7E5C0DE0001ull;

__device__ inline double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ inline void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// vectors b < 3 with use[b] (BS values at p[b]) into xv, lane l holding
// columns l, l + 32, ...: relaxed loads of the slots still holding the
// sentinel, repeated until the whole warp has every value. Bounded like
// flow_wait_n (ICX_FLOW_SPINS rounds, then *err = 1; a set *err ends it).
template <int BS, int NS, class TA>
__device__ inline bool flow_gather_ready(const double* p0, const double* p1, const double* p2, bool u0, bool u1,
                                         bool u2, TA (&xv)[3][NS], int* err) {
  const int lane = threadIdx.x & 31;
  const double* p[3] = {p0, p1, p2};
  const bool use[3] = {u0, u1, u2};
  unsigned pending = 0;
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      xv[b][s] = TA(0);
      if (use[b] && lane + 32 * s < BS) pending |= 1u << (b * NS + s);
    }
  unsigned spins = 0;
  while (true) {
    double v[3][NS];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int s = 0; s < NS; ++s)
        if (pending & (1u << (b * NS + s))) v[b][s] = ld_relaxed_f64(p[b] + lane + 32 * s);
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const unsigned bit = 1u << (b * NS + s);
        if ((pending & bit) && (unsigned long long)__double_as_longlong(v[b][s]) != FLOW_SENTINEL) {
          xv[b][s] = (TA)v[b][s];
          pending &= ~bit;
        }
      }
    if (__all_sync(0xffffffffu, pending == 0)) return true;
    int stop = 0;
    if (lane == 0) {
      if (*reinterpret_cast<volatile int*>(err)) stop = 1;
      else if (++spins > ICX_FLOW_SPINS) {
        atomicExch(err, 1);
        stop = 1;
      }
    }
    if (__shfl_sync(0xffffffffu, stop, 0)) return false;
  }
}

// an output value of the sentinel schedule (never the sentinel itself)
__device__ inline double flow_value(double v) {
  return (unsigned long long)__double_as_longlong(v) == FLOW_SENTINEL ? __longlong_as_double(0x7FFFFFFFFFFFFFFFll) : v;
}

// rows per task of the data-flow apply: three blocks' rows stay in registers.
// RT = 0 takes the block size's default; the others are tile choices (every
// row's sum is formed the same way whatever the rows per task)
// whether a task of r rows fits: at most the block size, and r x (values
// per lane per row) <= 24 register values
constexpr bool flow_rows_fit(int bs, int ns, int r) { return r <= (bs < 2 ? 2 : bs) && r * ns <= 24; }

template <int BS, int RT = 0>
struct FlowCfg {
  static constexpr int NS = (BS + 31) / 32;
  // default rows per task, measured (ms per apply): 64 x 64 blocks 1.15 with
  // 6 rows against 1.31 with 8 and 1.36 with 12; 36 x 36 blocks 2.40 with 4
  // against 2.48 with 6 and 3.71 with 2
  static constexpr int R_DEFAULT = NS >= 3 ? 4 : (BS >= 64 ? 6 : (BS >= 32 ? 4 : 2));
  static constexpr int R = RT ? RT : R_DEFAULT;
  static constexpr int GROUPS = (BS + R - 1) / R;
};

// SEN: the sentinel schedule (outputs pre-filled with FLOW_SENTINEL; the
// counters, epoch and flow_signal are not used), else completion counters
template <int BS, int RT, class TA, bool SEN>
__global__ void __launch_bounds__(256) ilu_apply_flow_kernel(IluFlowArgs<TA> a) {
  using K = FlowCfg<BS, RT>;
  constexpr int NS = K::NS, R = K::R, GROUPS = K::GROUPS;
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const long long ntask = (long long)a.E * GROUPS;
  const unsigned target = a.epoch * (unsigned)GROUPS;
  for (int sweep = 0; sweep < 2; ++sweep) {
    const bool fwd = sweep == 0;
    for (long long t = gw; t < ntask; t += nw) {
      if (*reinterpret_cast<volatile int*>(a.err)) return;
      const long long p = t / GROUPS;
      const int g = (int)(t - p * GROUPS);
      const int e = a.order[fwd ? p : a.E - 1 - p];
      const int r0 = g * R;
      // neighbour blocks: forward reads the strictly lower ones, backward the
      // strictly upper ones (at most two of each on quadrilateral meshes).
      // Indices are checked before use: a bad one sets *err = 2 and ends the
      // launch (the values are uniform over the warp, so the whole warp leaves).
      int nbk = 0, kbs[2], ks[2];
      bool bad = e < 0 || e >= a.E;
      if (!bad) {
        const int d = a.diag[e], rb = a.rowptr[e], re = a.rowptr[e + 1];
        bad = d < rb || d >= re || rb < 0 || re > a.nnzb;
        const int b0 = fwd ? rb : d + 1, b1 = fwd ? d : re;
        bad = bad || (b1 - b0) > 2;
        for (int kb = b0; !bad && kb < b1; ++kb) {
          kbs[nbk] = kb;
          ks[nbk] = a.colidx[kb];
          bad = ks[nbk] < 0 || ks[nbk] >= a.E;
          ++nbk;
        }
      }
      if (bad) {
        if (lane == 0) atomicExch(a.err, 2);
        return;
      }
      // matrix rows first: they do not depend on other tasks
      TA am[3][R][NS];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const TA* Ab = nullptr;
        if (b < 2 && b < nbk) Ab = a.LU + (size_t)kbs[b] * BS * BS;
        else if (b == 2 && !fwd) Ab = a.Uinv + (size_t)e * BS * BS;
#pragma unroll
        for (int rr = 0; rr < R; ++rr)
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            const int r = r0 + rr, c = lane + 32 * s;
            am[b][rr][s] = (Ab && r < BS && c < BS) ? Ab[(size_t)r * BS + c] : TA(0);
          }
      }
      TA acc[R];
#pragma unroll
      for (int rr = 0; rr < R; ++rr) acc[rr] = TA(0);
      const double* vsrc = fwd ? a.f : a.y;
      unsigned* cnt = fwd ? a.cnt_f : a.cnt_b;
      TA xv[3][NS];
      if constexpr (SEN) {
        // the neighbours' rows (backward: and the element's own forward
        // result) as soon as none of them holds the sentinel
        if (!flow_gather_ready<BS, NS, TA>(vsrc + (size_t)(nbk > 0 ? ks[0] : 0) * BS,
                                           vsrc + (size_t)(nbk > 1 ? ks[1] : 0) * BS, a.f + (size_t)e * BS,
                                           nbk > 0, nbk > 1, !fwd, xv, a.err))
          return;
      } else {
        // every dependency first (backward: also the element's own forward
        // result), then all the vectors in one round of loads, so that the
        // second neighbour's load does not add another L2 round trip
        {
          // counters: the nbk neighbours, then (backward) the element's own forward one
          const unsigned* w0 = nbk > 0 ? cnt + ks[0] : a.cnt_f + e;
          const unsigned* w1 = nbk > 1 ? cnt + ks[1] : a.cnt_f + e;
          const int nw = nbk + (fwd ? 0 : 1);
          if (nw > 0 && !flow_wait_n(w0, w1, a.cnt_f + e, nw, target, a.err)) return;
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int c = lane + 32 * s;
#pragma unroll
          for (int b = 0; b < 2; ++b) xv[b][s] = (b < nbk && c < BS) ? (TA)__ldcg(vsrc + (size_t)ks[b] * BS + c) : TA(0);
          xv[2][s] = (!fwd && c < BS) ? (TA)__ldcg(a.f + (size_t)e * BS + c) : TA(0);
        }
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (b < nbk) {
#pragma unroll
          for (int rr = 0; rr < R; ++rr)
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[rr] = fused_madd(-am[b][rr][s], xv[b][s], acc[rr]);
        }
      }
      if (!fwd) {
        // y_e = inv(U_ee) f_e + acc
#pragma unroll
        for (int rr = 0; rr < R; ++rr)
#pragma unroll
          for (int s = 0; s < NS; ++s) acc[rr] = fused_madd(am[2][rr][s], xv[2][s], acc[rr]);
      }
      const RowSum<TA> rs = warp_row_sums<R>(acc);
      const TA mine = rs.v;
      const int r = r0 + rs.row;
      if constexpr (SEN) {
        if (rs.owner && r < BS) {
          if (fwd) st_relaxed_f64(a.f + (size_t)e * BS + r, flow_value(a.x[(size_t)e * BS + r] + (double)mine));
          else st_relaxed_f64(a.y + (size_t)e * BS + r, flow_value((double)mine));
        }
      } else {
        if (rs.owner && r < BS) {
          if (fwd) a.f[(size_t)e * BS + r] = a.x[(size_t)e * BS + r] + (double)mine;
          else a.y[(size_t)e * BS + r] = (double)mine;
        }
        flow_signal(cnt + e);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Block-ILU(0) apply on element groups (tiles): one CTA per group. A group's
// factors couple none of its elements to another group, so its two sweeps
// need nothing from outside it: the CTA runs its elements level by level
// (levels of the kept lower dependencies, ascending for the forward sweep,
// descending for the backward one), the tasks of one level (element, R rows)
// spread over its warps, with a CTA barrier between levels. A task reads the
// results of earlier levels with ordinary loads: the barrier orders the
// CTA's own stores before them. No cross-CTA waits, so no polling.
struct IluGroupPlan {
  int ngroups;
  const int4* task;     // [2 E] per position in the group order: {element, first block, k0, k1} of its
                        // forward (first E) and backward (last E) sweep rows; k = -1: no such block
  const int* glev;      // level boundaries: positions in the group order, group g's at glev[glev_ptr[g] .. glev_ptr[g + 1]]
  const int* glev_ptr;  // [ngroups + 1]
  int gmax;             // elements of the largest group
  const int4* loc;      // [2 E] the same entries by position within the group: {element, k0, k1, 0}
                        // (ilu_apply_group_rows_kernel only)
};

template <class TA>
struct IluGroupArgs {
  int E, nnzb;
  const TA* LU;
  const TA* Uinv;
  const double* x;
  double* f;            // forward result (written and read by the group's own CTA)
  double* y;            // output
  int* err;
  IluGroupPlan plan;
};

// threads per CTA of the group applies by default: FP32 factors keep their
// rows in half the registers, so twice the warps fit a CTA
template <class TA>
constexpr int group_threads() { return sizeof(TA) == 8 ? 256 : 512; }

// levels of a group kept in shared memory (more: read from global memory)
constexpr int kGroupLevelsSmem = 256;

// one task: rows r0 .. r0 + R - 1 of the element's sweep row, with the same
// arithmetic in the same order as the data-flow apply:
// f_e = x_e - sum L_ek f_k; y_e = inv(U_ee) f_e - sum (inv(U_ee) U_ek) y_k
template <int BS, int R, int NS, class TA>
__device__ inline void group_task_run(const IluGroupArgs<TA>& a, bool fwd, int4 inf, int r0) {
  const int lane = threadIdx.x & 31;
  const int e = inf.x, b0 = inf.y, k0 = inf.z, k1 = inf.w;
  const int nbk = (k0 >= 0) + (k1 >= 0);
  const bool bad = e < 0 || e >= a.E || b0 < 0 || b0 + nbk > a.nnzb || k0 >= a.E || k1 >= a.E || (k1 >= 0 && k0 < 0);
  if (bad) {  // uniform over the warp
    if (lane == 0) atomicExch(a.err, 2);
    return;
  }
  TA am[3][R][NS];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const TA* Ab = nullptr;
    if (b < 2 && b < nbk) Ab = a.LU + (size_t)(b0 + b) * BS * BS;
    else if (b == 2 && !fwd) Ab = a.Uinv + (size_t)e * BS * BS;
#pragma unroll
    for (int rr = 0; rr < R; ++rr)
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int r = r0 + rr, c = lane + 32 * s;
        am[b][rr][s] = (Ab && r < BS && c < BS) ? Ab[(size_t)r * BS + c] : TA(0);
      }
  }
  const double* vsrc = fwd ? a.f : a.y;
  TA xv[3][NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int c = lane + 32 * s;
    xv[0][s] = (nbk > 0 && c < BS) ? (TA)vsrc[(size_t)k0 * BS + c] : TA(0);
    xv[1][s] = (nbk > 1 && c < BS) ? (TA)vsrc[(size_t)k1 * BS + c] : TA(0);
    xv[2][s] = (!fwd && c < BS) ? (TA)a.f[(size_t)e * BS + c] : TA(0);
  }
  TA acc[R];
#pragma unroll
  for (int rr = 0; rr < R; ++rr) acc[rr] = TA(0);
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    if (b < nbk) {
#pragma unroll
      for (int rr = 0; rr < R; ++rr)
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[rr] = fused_madd(-am[b][rr][s], xv[b][s], acc[rr]);
    }
  }
  if (!fwd) {
#pragma unroll
    for (int rr = 0; rr < R; ++rr)
#pragma unroll
      for (int s = 0; s < NS; ++s) acc[rr] = fused_madd(am[2][rr][s], xv[2][s], acc[rr]);
  }
  const RowSum<TA> rs = warp_row_sums<R>(acc);
  const TA mine = rs.v;
  const int r = r0 + rs.row;
  if (rs.owner && r < BS) {
    if (fwd) a.f[(size_t)e * BS + r] = a.x[(size_t)e * BS + r] + (double)mine;
    else a.y[(size_t)e * BS + r] = (double)mine;
  }
}

// the group's levels in sweep order: q < nlev forward level q, then the
// backward levels from the last one down. Each warp's tasks of a level are
// t = warp, warp + nwarp, ...; the task-table entry of a warp's next task
// (in this level or, after its last one, its first of the next level) is
// loaded before the current task runs, so a task costs one dependent trip
// to memory (its matrix rows and neighbour vectors, loaded together)
template <int BS, int RT, class TA, int NT>
__global__ void __launch_bounds__(NT) ilu_apply_group_kernel(IluGroupArgs<TA> a) {
  using K = FlowCfg<BS, RT>;
  constexpr int NS = K::NS, R = K::R, GROUPS = K::GROUPS;
  __shared__ int slev[kGroupLevelsSmem + 1];
  const int warp = threadIdx.x >> 5, nwarp = NT / 32;
  const int g = blockIdx.x;
  const int l0 = a.plan.glev_ptr[g], l1 = a.plan.glev_ptr[g + 1];
  const int nlev = l1 - l0 - 1;
  const bool in_smem = nlev <= kGroupLevelsSmem;
  if (in_smem)
    for (int i = threadIdx.x; i <= nlev; i += blockDim.x) slev[i] = a.plan.glev[l0 + i];
  __syncthreads();
  auto lev = [&](int i) { return in_smem ? slev[i] : a.plan.glev[l0 + i]; };
  const int nq = 2 * nlev;
  int4 inf = make_int4(-1, 0, -1, -1);
  bool have = false;
  for (int q = 0; q < nq; ++q) {
    const bool fwd = q < nlev;
    const int lv = fwd ? q : nq - 1 - q;
    const int p0 = lev(lv), ntask = (lev(lv + 1) - p0) * GROUPS;
    const int4* tk = a.plan.task + (fwd ? 0 : a.E);
    if (!have && warp < ntask) inf = tk[p0 + warp / GROUPS];
    have = false;
    for (int t = warp; t < ntask; t += nwarp) {
      int4 nxt = inf;
      const int tn = t + nwarp;
      if (tn < ntask) {
        nxt = tk[p0 + tn / GROUPS];
        have = true;
      } else if (q + 1 < nq) {
        const bool fn = q + 1 < nlev;
        const int ln = fn ? q + 1 : nq - 2 - q;
        const int pn = lev(ln), nn = (lev(ln + 1) - pn) * GROUPS;
        if (warp < nn) {
          nxt = a.plan.task[(fn ? 0 : a.E) + pn + warp / GROUPS];
          have = true;
        }
      }
      group_task_run<BS, R, NS, TA>(a, fwd, inf, (t % GROUPS) * R);
      inf = nxt;
    }
    __syncthreads();
  }
}

// the group apply with the matrix rows staged in shared memory: each warp
// copies the rows of its next D tasks (cp.async, no registers held) into its
// own ring of D slots while it runs the current one, across level barriers
// (the factors are read-only), so a task waits only for its neighbours'
// vectors; the group's task-table entries are staged once at the start.
// Dynamic shared memory: 2 gmax entries (int4), then nwarp x D slots of
// group_slot_bytes<BS, R, TA>() bytes. Same arithmetic in the same order as
// ilu_apply_group_kernel (bit-identical results).
template <int BS, int R, class TA>
__host__ __device__ constexpr int group_slot_bytes() {
  return ((3 * R * BS * (int)sizeof(TA)) + 15) / 16 * 16;
}

__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// copies n bytes (a multiple of CH, both addresses CH-aligned) over the warp
template <int CH>
__device__ inline void cp_async_span(void* sdst, const void* gsrc, int n) {
  const int lane = threadIdx.x & 31;
  const unsigned d0 = (unsigned)__cvta_generic_to_shared(sdst);
  const char* s0 = (const char*)gsrc;
  for (int o = lane * CH; o < n; o += 32 * CH) {
    if constexpr (CH == 16)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d0 + o), "l"(s0 + o) : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d0 + o), "l"(s0 + o), "n"(CH) : "memory");
  }
}

template <int BS, int R, class TA>
__device__ inline bool group_task_ok(const IluGroupArgs<TA>& a, int4 inf) {
  const int nbk = (inf.z >= 0) + (inf.w >= 0);
  return !(inf.x < 0 || inf.x >= a.E || inf.y < 0 || inf.y + nbk > a.nnzb || inf.z >= a.E || inf.w >= a.E ||
           (inf.w >= 0 && inf.z < 0));
}

template <int BS, int RT, class TA, int NT, int D>
__global__ void __launch_bounds__(NT) ilu_apply_group_async_kernel(IluGroupArgs<TA> a) {
  using K = FlowCfg<BS, RT>;
  constexpr int NS = K::NS, R = K::R, GROUPS = K::GROUPS;
  constexpr int SLOT = group_slot_bytes<BS, R, TA>();
  constexpr int CH = (BS * (int)sizeof(TA)) % 16 == 0 ? 16 : (int)sizeof(TA);
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ int slev[kGroupLevelsSmem + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = NT / 32;
  const int g = blockIdx.x;
  const int l0 = a.plan.glev_ptr[g], l1 = a.plan.glev_ptr[g + 1];
  const int nlev = l1 - l0 - 1;
  const int pg0 = a.plan.glev[l0], G = a.plan.glev[l1 - 1] - pg0;
  // the launch guarantees G <= gmax and nlev <= kGroupLevelsSmem; a plan
  // that breaks either is reported, not run
  if (nlev > kGroupLevelsSmem || G > a.plan.gmax || G < 0) {
    if (threadIdx.x == 0) atomicExch(a.err, 2);
    return;
  }
  int4* sinfo = reinterpret_cast<int4*>(dsm);
  unsigned char* ring = dsm + (size_t)2 * a.plan.gmax * sizeof(int4) + (size_t)warp * D * SLOT;
  for (int i = threadIdx.x; i <= nlev; i += blockDim.x) slev[i] = a.plan.glev[l0 + i];
  for (int i = threadIdx.x; i < G; i += blockDim.x) {
    sinfo[i] = a.plan.task[pg0 + i];
    sinfo[G + i] = a.plan.task[a.E + pg0 + i];
  }
  __syncthreads();
  const int nq = 2 * nlev;
  auto ntask = [&](int q) {
    const int lv = q < nlev ? q : nq - 1 - q;
    return (slev[lv + 1] - slev[lv]) * GROUPS;
  };
  auto info = [&](int q, int t) {
    const bool fwd = q < nlev;
    const int lv = fwd ? q : nq - 1 - q;
    return sinfo[(fwd ? 0 : G) + slev[lv] - pg0 + t / GROUPS];
  };
  // the issue cursor: the warp's next task whose rows are not yet requested
  int qi = 0, ti = warp;
  while (qi < nq && ti >= ntask(qi)) ++qi;
  auto issue = [&](int slot) {
    if (qi < nq) {
      const bool fwd = qi < nlev;
      const int4 inf = info(qi, ti);
      if (group_task_ok<BS, R, TA>(a, inf)) {
        const int r0 = (ti % GROUPS) * R;
        const int nr = BS - r0 < R ? BS - r0 : R;
        const int nbk = (inf.z >= 0) + (inf.w >= 0);
        unsigned char* dst = ring + (size_t)slot * SLOT;
        for (int b = 0; b < 3; ++b) {
          const TA* src = nullptr;
          if (b < 2 && b < nbk) src = a.LU + (size_t)(inf.y + b) * BS * BS;
          else if (b == 2 && !fwd) src = a.Uinv + (size_t)inf.x * BS * BS;
          if (src) cp_async_span<CH>(dst + (size_t)b * R * BS * sizeof(TA), src + (size_t)r0 * BS,
                                     nr * BS * (int)sizeof(TA));
        }
      }
      ti += nwarp;
      while (qi < nq && ti >= ntask(qi)) {
        ++qi;
        ti = warp;
      }
    }
    cp_async_commit();  // possibly empty: one group per task keeps the count
  };
#pragma unroll
  for (int d = 0; d < D; ++d) issue(d);
  int n = 0;
  for (int q = 0; q < nq; ++q) {
    const bool fwd = q < nlev;
    const int nt = ntask(q);
    for (int t = warp; t < nt; t += nwarp, ++n) {
      cp_async_wait<D - 1>();
      __syncwarp();
      const int4 inf = info(q, t);
      const int slot = n % D;
      if (!group_task_ok<BS, R, TA>(a, inf)) {
        if (lane == 0) atomicExch(a.err, 2);
      } else {
        const TA* am = reinterpret_cast<const TA*>(ring + (size_t)slot * SLOT);
        const int e = inf.x, k0 = inf.z, k1 = inf.w, r0 = (t % GROUPS) * R;
        const int nbk = (k0 >= 0) + (k1 >= 0);
        const double* vsrc = fwd ? a.f : a.y;
        TA xv[3][NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int c = lane + 32 * s;
          xv[0][s] = (nbk > 0 && c < BS) ? (TA)vsrc[(size_t)k0 * BS + c] : TA(0);
          xv[1][s] = (nbk > 1 && c < BS) ? (TA)vsrc[(size_t)k1 * BS + c] : TA(0);
          xv[2][s] = (!fwd && c < BS) ? (TA)a.f[(size_t)e * BS + c] : TA(0);
        }
        auto mat = [&](int b, int rr, int s) {
          const int c = lane + 32 * s;
          return (r0 + rr < BS && c < BS) ? am[(b * R + rr) * BS + c] : TA(0);
        };
        TA acc[R];
#pragma unroll
        for (int rr = 0; rr < R; ++rr) acc[rr] = TA(0);
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          if (b < nbk) {
#pragma unroll
            for (int rr = 0; rr < R; ++rr)
#pragma unroll
              for (int s = 0; s < NS; ++s) acc[rr] = fused_madd(-mat(b, rr, s), xv[b][s], acc[rr]);
          }
        }
        if (!fwd) {
#pragma unroll
          for (int rr = 0; rr < R; ++rr)
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[rr] = fused_madd(mat(2, rr, s), xv[2][s], acc[rr]);
        }
        const RowSum<TA> rs = warp_row_sums<R>(acc);
        const TA mine = rs.v;
        const int r = r0 + rs.row;
        if (rs.owner && r < BS) {
          if (fwd) a.f[(size_t)e * BS + r] = a.x[(size_t)e * BS + r] + (double)mine;
          else a.y[(size_t)e * BS + r] = (double)mine;
        }
      }
      __syncwarp();  // the slot is read by every lane before it is refilled
      issue(slot);
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

// The group apply with one lane per matrix row: the tasks of a level are
// its (element, row) pairs, 32 to a warp, and a lane forms its row's sums
// over the columns in order, reading the factor row with the widest loads
// (up to 16 bytes) its alignment allows. The group's forward and backward
// vectors stay in shared memory (rounded to the arithmetic type, as the
// other applies round them on load), so a task's only reads from memory are
// its factor rows and x; the forward vector is not written back. No warp
// reductions. The column order of the sums differs from the other applies
// (not bit-identical to them; identical across thread counts). TS is the
// factors' storage type: double and float are also the arithmetic type,
// BF16 factors are widened to FP32. Dynamic shared memory: 4 gmax entries
// (int4), then 2 gmax BS values of the arithmetic type.
template <class TS>
struct ComputeOf {
  using type = TS;
};
template <>
struct ComputeOf<__nv_bfloat16> {
  using type = float;
};

// bytes per factor-row load: the widest of 16 / 8 / 4 / 2 dividing a row
template <int BS, class TS>
__host__ __device__ constexpr int group_rows_load_bytes() {
  constexpr int row = BS * (int)sizeof(TS);
  return row % 16 == 0 ? 16 : row % 8 == 0 ? 8 : row % 4 == 0 ? 4 : (int)sizeof(TS);
}

template <class TC>
__host__ __device__ constexpr size_t group_rows_smem(int gmax, int bs) {
  return (size_t)4 * gmax * sizeof(int4) + (size_t)2 * gmax * bs * sizeof(TC);
}

template <int BYTES>
struct RawLoad;
template <> struct RawLoad<16> { using type = uint4; };
template <> struct RawLoad<8> { using type = uint2; };
template <> struct RawLoad<4> { using type = unsigned; };
template <> struct RawLoad<2> { using type = unsigned short; };

template <class TS>
__device__ inline typename ComputeOf<TS>::type widen(TS v) {
  if constexpr (std::is_same<TS, __nv_bfloat16>::value) return __bfloat162float(v);
  else return v;
}

// one factor row, held in registers (all its loads issued before any use)
template <int BS, class TS>
struct FactorRow {
  using TC = typename ComputeOf<TS>::type;
  static constexpr int LB = group_rows_load_bytes<BS, TS>();
  static constexpr int VEC = LB / (int)sizeof(TS);  // factor values per load
  using V = typename RawLoad<LB>::type;
  V v[BS / VEC];
  __device__ inline void load(const TS* __restrict__ arow) {
#pragma unroll
    for (int c = 0; c < BS / VEC; ++c) v[c] = __ldg(reinterpret_cast<const V*>(arow) + c);
  }
  // acc += sign * row . x over the BS columns, in column order (x in shared
  // memory, arithmetic type)
  template <bool NEG>
  __device__ inline TC dot(const TC* xs, TC acc) const {
#pragma unroll
    for (int c = 0; c < BS / VEC; ++c) {
      const TS* av = reinterpret_cast<const TS*>(&v[c]);
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        const TC aw = widen(av[i]);
        acc = fused_madd(NEG ? -aw : aw, xs[c * VEC + i], acc);
      }
    }
    return acc;
  }
};

template <int BS, class TS, int NT>
__global__ void __launch_bounds__(NT) ilu_apply_group_rows_kernel(IluGroupArgs<TS> a) {
  using TC = typename ComputeOf<TS>::type;
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ int slev[kGroupLevelsSmem + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = blockIdx.x;
  const int l0 = a.plan.glev_ptr[g], l1 = a.plan.glev_ptr[g + 1];
  const int nlev = l1 - l0 - 1;
  const int gm = a.plan.gmax;
  const int pg0 = a.plan.glev[l0], G = a.plan.glev[l1 - 1] - pg0;
  if (nlev > kGroupLevelsSmem || G > gm || G < 0) {  // uniform over the CTA
    if (threadIdx.x == 0) atomicExch(a.err, 2);
    return;
  }
  int4* sinfo = reinterpret_cast<int4*>(dsm);  // [fwd gmax | bwd gmax]
  int4* sloc = sinfo + 2 * gm;                 // [fwd gmax | bwd gmax]
  TC* fs = reinterpret_cast<TC*>(sloc + 2 * gm);
  TC* ys = fs + (size_t)gm * BS;
  for (int i = threadIdx.x; i <= nlev; i += NT) slev[i] = a.plan.glev[l0 + i];
  for (int i = threadIdx.x; i < G; i += NT) {
    sinfo[i] = a.plan.task[pg0 + i];
    sinfo[gm + i] = a.plan.task[a.E + pg0 + i];
    sloc[i] = a.plan.loc[pg0 + i];
    sloc[gm + i] = a.plan.loc[a.E + pg0 + i];
  }
  __syncthreads();
  const int nq = 2 * nlev;
  for (int q = 0; q < nq; ++q) {
    const bool fwd = q < nlev;
    const int lv = fwd ? q : nq - 1 - q;
    const int p0 = slev[lv] - pg0, npair = (slev[lv + 1] - slev[lv]) * BS;
    const int4* ti = sinfo + (fwd ? 0 : gm);
    const int4* tl = sloc + (fwd ? 0 : gm);
    for (int t = warp; t * 32 < npair; t += NW) {
      const int p = t * 32 + lane;
      if (p >= npair) continue;
      const int ei = p / BS, r = p - ei * BS;
      const int4 inf = ti[p0 + ei], loc = tl[p0 + ei];
      const int nbk = (inf.z >= 0) + (inf.w >= 0);
      const bool bad = !group_task_ok<BS, 1, TS>(a, inf) || loc.x < 0 || loc.x >= G || loc.y >= G ||
                       loc.z >= G || (nbk > 0 && loc.y < 0) || (nbk > 1 && loc.z < 0);
      if (bad) {
        atomicExch(a.err, 2);
        continue;
      }
      TC acc = TC(0);
      const TC* xs = fwd ? fs : ys;
      // both off-diagonal rows in flight together (the second block's row
      // loads the diagonal inverse's row on a backward row with one block)
      FactorRow<BS, TS> r0, r1;
      if (nbk > 0) r0.load(a.LU + ((size_t)inf.y * BS + r) * BS);
      if (nbk > 1) r1.load(a.LU + ((size_t)(inf.y + 1) * BS + r) * BS);
      else if (!fwd) r1.load(a.Uinv + ((size_t)inf.x * BS + r) * BS);
      const double xe = fwd ? a.x[(size_t)inf.x * BS + r] : 0.0;
      if (nbk > 0) acc = r0.template dot<true>(xs + (size_t)loc.y * BS, acc);
      if (nbk > 1) {
        acc = r1.template dot<true>(xs + (size_t)loc.z * BS, acc);
        if (!fwd) r1.load(a.Uinv + ((size_t)inf.x * BS + r) * BS);
      }
      if (fwd) {
        const double fd = xe + (double)acc;
        fs[(size_t)loc.x * BS + r] = (TC)fd;
      } else {
        acc = r1.template dot<false>(fs + (size_t)loc.x * BS, acc);
        a.y[(size_t)inf.x * BS + r] = (double)acc;
        ys[(size_t)loc.x * BS + r] = acc;
      }
    }
    __syncthreads();
  }
}

#define ICX_BLOCK_SIZES(X) X(4) X(9) X(16) X(25) X(36) X(64) X(100)

}  // namespace icx
