// Launch-shape autotuner. The tunable kernels are compiled in several launch
// shapes (TileChoice) that move work between threads, warps and CTAs without
// changing any value or summation order:
//   face_flux_kernel      the register bound's resident CTAs per SM
//   vol_lift_kernel       threads per CTA (and so elements per CTA) and its register bound
//   ilu_apply_flow_kernel block rows per warp task, CTAs per SM and the schedule
//                         (completion counters or sentinel values; FP64 and FP32 factors)
// icx_autotune times each shape on the context's own mesh and state with CUDA
// events, flushing L2 before every timed launch as the benchmarks do, checks
// that its output equals the default shape's bit for bit (a shape that
// differs is rejected and counted), and keeps the fastest. Choices are cached
// per process under the key (dimension, p, neq, geometry order, viscous flux).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "icx_internal.h"

namespace {

using icx::TileChoice;

constexpr int TUNE_ALL = ICX_TUNE_RESIDUAL | ICX_TUNE_ILU | ICX_TUNE_ILU_FP32;
constexpr int REPS = 7;                        // timed launches per candidate (median)
constexpr size_t FLUSH_BYTES = 256ull << 20;   // written before every timed launch (L2 is 126 MB)
constexpr int MAX_CTAS = 4;                    // CTAs per SM tried for the ILU apply
constexpr double MARGIN = 0.99;                // a shape replaces the best so far only when 1 % faster

struct CacheEntry {
  TileChoice tile;
  int parts = 0;  // ICX_TUNE_* bits whose fields hold a tuned choice
};
// dim, p, neq, geometry order, DDG flux, and the block-ILU(0) tiling the
// apply was timed on (tile side, 0 untiled, -1 element groups)
using Key = std::tuple<int, int, int, int, int, int>;
std::mutex g_mu;
std::map<Key, CacheEntry> g_cache;

icx_status fail(icx_ctx* c, icx_status st, const std::string& m) {
  if (c) c->err = m;
  return st;
}

#define TCK(expr)                                                                                     \
  do {                                                                                                \
    cudaError_t _e = (expr);                                                                          \
    if (_e != cudaSuccess) return fail(c, ICX_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

__global__ void count_diff_kernel(const unsigned long long* __restrict__ a, const unsigned long long* __restrict__ b,
                                  long long n, unsigned long long* count) {
  unsigned long long local = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    local += a[i] != b[i];
  if (local) atomicAdd(count, local);
}

// a fixed right-hand side in [-1, 1): a 64-bit integer hash of the index
__global__ void fill_hash_kernel(double* x, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    x[i] = (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// device scratch of one tuning call, released on every exit path
struct Scratch {
  std::vector<void*> ptrs;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
  template <class T>
  cudaError_t alloc(T** p, size_t bytes) {
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

struct Tuner {
  icx_ctx* c = nullptr;
  Scratch sc;
  void* flush = nullptr;
  unsigned long long* diff = nullptr;
  cudaStream_t s = 0;
  int timed = 0, rejected = 0;

  icx_status init() {
    TCK(sc.alloc(&flush, FLUSH_BYTES));
    TCK(sc.alloc(&diff, sizeof(unsigned long long)));
    TCK(cudaEventCreate(&sc.ev[0]));
    TCK(cudaEventCreate(&sc.ev[1]));
    return ICX_OK;
  }

  // median device time of op over REPS launches, L2 flushed before each
  template <class Op>
  icx_status time(Op op, double* ms) {
    std::vector<float> t(REPS);
    for (int r = 0; r < REPS; ++r) {
      TCK(cudaMemsetAsync(flush, r & 0xff, FLUSH_BYTES, s));
      TCK(cudaEventRecord(sc.ev[0], s));
      TCK(op());
      TCK(cudaEventRecord(sc.ev[1], s));
      TCK(cudaEventSynchronize(sc.ev[1]));
      TCK(cudaEventElapsedTime(&t[r], sc.ev[0], sc.ev[1]));
    }
    std::sort(t.begin(), t.end());
    *ms = t[REPS / 2];
    ++timed;
    return ICX_OK;
  }

  // number of 64-bit words in which a and b differ
  icx_status differ(const double* a, const double* b, long long n, unsigned long long* out) {
    TCK(cudaMemsetAsync(diff, 0, sizeof(unsigned long long), s));
    count_diff_kernel<<<592, 256, 0, s>>>(reinterpret_cast<const unsigned long long*>(a),
                                          reinterpret_cast<const unsigned long long*>(b), n, diff);
    TCK(cudaGetLastError());
    TCK(cudaMemcpyAsync(out, diff, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    TCK(cudaStreamSynchronize(s));
    return ICX_OK;
  }

  // face and volume kernels: the face bound first (volume default), then the
  // volume tile with the chosen face bound
  icx_status residual(const double* u, double* ms_def, double* ms_tuned) {
    icx::DeviceMesh& dm = c->dm;
    const long long n = (long long)dm.E * dm.nb * dm.neq;
    double *r0 = nullptr, *r1 = nullptr;
    TCK(sc.alloc(&r0, sizeof(double) * n));
    TCK(sc.alloc(&r1, sizeof(double) * n));
    const TileChoice keep = dm.tile;
    dm.tile.face_minb = 0;
    dm.tile.vol_threads = dm.tile.vol_minb = 0;
    auto run = [&](double* out) { return icx::launch_residual(dm, c->phys, u, out, s); };
    TCK(run(r0));
    TCK(cudaStreamSynchronize(s));
    icx_status st = time([&] { return run(r1); }, ms_def);
    if (st != ICX_OK) { dm.tile = keep; return st; }
    const int D = icx::face_minb_default(c->phys.pde, c->phys.beta1 != 0.0);
    double best = *ms_def;
    int best_face = D;
    for (int mb : {D - 1, D + 1}) {
      dm.tile.face_minb = mb;
      double ms = 0;
      unsigned long long nd = 0;
      if (run(r1) != cudaSuccess) { st = fail(c, ICX_ERR_CUDA, "residual tile launch failed"); break; }
      if ((st = differ(r0, r1, n, &nd)) != ICX_OK) break;
      if (nd) { ++rejected; continue; }
      if ((st = time([&] { return run(r1); }, &ms)) != ICX_OK) break;
      if (ms < MARGIN * best) { best = ms; best_face = mb; }
    }
    if (st != ICX_OK) { dm.tile = keep; return st; }
    dm.tile.face_minb = best_face;
    int best_vol = 0;
    for (int i = 1; i < icx::kNumVolTiles; ++i) {
      dm.tile.vol_threads = icx::kVolTiles[i].threads;
      dm.tile.vol_minb = icx::kVolTiles[i].minb;
      double ms = 0;
      unsigned long long nd = 0;
      if (run(r1) != cudaSuccess) { st = fail(c, ICX_ERR_CUDA, "residual tile launch failed"); break; }
      if ((st = differ(r0, r1, n, &nd)) != ICX_OK) break;
      if (nd) { ++rejected; continue; }
      if ((st = time([&] { return run(r1); }, &ms)) != ICX_OK) break;
      if (ms < MARGIN * best) { best = ms; best_vol = i; }
    }
    if (st != ICX_OK) { dm.tile = keep; return st; }
    dm.tile.vol_threads = icx::kVolTiles[best_vol].threads;
    dm.tile.vol_minb = icx::kVolTiles[best_vol].minb;
    *ms_tuned = best;
    return ICX_OK;
  }

  // FD Jacobian at u, block-ILU(0) factors (FP64 and FP32), then every
  // (schedule, rows per task, CTAs per SM) of the requested precisions
  icx_status ilu(const double* u, bool fp64, bool fp32, double* ms_def, double* ms_tuned) {
    icx::DeviceMesh& dm = c->dm;
    const int bs = dm.nb * dm.neq;
    const long long n = (long long)dm.E * bs;
    double *vals = nullptr, *res = nullptr, *x = nullptr, *z0 = nullptr, *z1 = nullptr;
    TCK(sc.alloc(&vals, sizeof(double) * (size_t)dm.nnzb * bs * bs));
    TCK(sc.alloc(&res, sizeof(double) * n));
    TCK(sc.alloc(&x, sizeof(double) * n));
    TCK(sc.alloc(&z0, sizeof(double) * n));
    TCK(sc.alloc(&z1, sizeof(double) * n));
    TCK(icx::launch_jacobian_fd(dm, c->phys, u, res, vals, std::sqrt(DBL_EPSILON), s));
    fill_hash_kernel<<<592, 256, 0, s>>>(x, n);
    TCK(cudaGetLastError());
    TCK(cudaStreamSynchronize(s));
    icx_status st = icx::solver_prepare_pc(c, vals, 2, -1);
    if (st != ICX_OK) return st;
    for (int pi = 0; pi < 2; ++pi) {
      if (!(pi == 0 ? fp64 : fp32)) continue;
      const bool mixed = pi == 1;
      const TileChoice keep = dm.tile;
      auto apply = [&](double* out) { return icx::solver_apply_ilu_flow(c, mixed, x, out, s); };
      auto check_err = [&]() -> icx_status {
        int perr = 0;
        icx_status e2 = icx::solver_take_pc_err(c, &perr);
        if (e2 != ICX_OK) return e2;
        if (perr) return fail(c, ICX_ERR_CUDA, perr == 1 ? "ILU apply: a dependency wait timed out"
                                                          : "ILU apply: bad block index");
        return ICX_OK;
      };
      dm.tile.flow_rows[pi] = dm.tile.flow_ctas[pi] = dm.tile.flow_sched[pi] = 0;
      TCK(apply(z0));
      TCK(cudaStreamSynchronize(s));
      if ((st = check_err()) != ICX_OK) { dm.tile = keep; return st; }
      if ((st = time([&] { return apply(z1); }, &ms_def[pi])) != ICX_OK ||
          (st = check_err()) != ICX_OK) { dm.tile = keep; return st; }
      // tiled / grouped factors: the per-group applies (schedules 3 to 5,
      // whose launch has no CTAs-per-SM choice) are candidates, 5 (FP32) or
      // 4 (FP64) the default
      const bool grouped = c->ilu_tile != 0 || !c->ilu_groups.empty();
      const int R0 = icx::flow_rows_default(bs), S0 = grouped ? icx::group_sched_default(pi) : icx::kFlowSchedDefault;
      double best = ms_def[pi];
      int best_r = R0, best_c = 2, best_s = S0;
      for (int sc = 1; sc <= (grouped ? 5 : 2); ++sc)
      for (int r : icx::kFlowRows) {
        if (!icx::flow_rows_compiled(bs, r)) continue;
        for (int k = 1; k <= MAX_CTAS; ++k) {
          if (sc >= 3 && k > 3) continue;  // 512 / 256 / 128 threads per group CTA
          if (sc == 5 && r != R0) continue;  // one lane per row: no rows-per-task choice
          if (r == R0 && k == 2 && sc == S0) continue;  // the default, timed above
          dm.tile.flow_rows[pi] = r;
          dm.tile.flow_ctas[pi] = k;
          dm.tile.flow_sched[pi] = sc;
          double ms = 0;
          unsigned long long nd = 0;
          cudaError_t e = apply(z1);
          if (e == cudaSuccess) e = cudaStreamSynchronize(s);
          if (e != cudaSuccess) { dm.tile = keep; return fail(c, ICX_ERR_CUDA, std::string("ILU tile: ") + cudaGetErrorString(e)); }
          if ((st = check_err()) != ICX_OK || (st = differ(z0, z1, n, &nd)) != ICX_OK) { dm.tile = keep; return st; }
          if (nd) { ++rejected; continue; }
          if ((st = time([&] { return apply(z1); }, &ms)) != ICX_OK || (st = check_err()) != ICX_OK) {
            dm.tile = keep;
            return st;
          }
          if (ms < MARGIN * best) { best = ms; best_r = r; best_c = k; best_s = sc; }
        }
      }
      dm.tile.flow_rows[pi] = best_r;
      dm.tile.flow_ctas[pi] = best_c;
      dm.tile.flow_sched[pi] = best_s;
      ms_tuned[pi] = best;
    }
    return ICX_OK;
  }
};

void to_public(const TileChoice& t, icx_tile_choice* o) {
  o->face_minb = t.face_minb;
  o->vol_threads = t.vol_threads;
  o->vol_minb = t.vol_minb;
  for (int k = 0; k < 2; ++k) {
    o->ilu_rows[k] = t.flow_rows[k];
    o->ilu_ctas[k] = t.flow_ctas[k];
    o->ilu_sched[k] = t.flow_sched[k];
  }
}

Key key_of(const icx_ctx* c) {
  return Key{2, c->dm.P, c->dm.neq, c->dm.G, c->phys.beta1 != 0.0 ? 1 : 0,
             c->ilu_groups.empty() ? c->ilu_tile : -1};
}

}  // namespace

extern "C" {

icx_status icx_tile_get(const icx_ctx* c, icx_tile_choice* t) {
  if (!c || !t) return ICX_ERR_INVALID;
  to_public(c->dm.tile, t);
  return ICX_OK;
}

icx_status icx_tile_set(icx_ctx* c, const icx_tile_choice* t) {
  if (!c || !t) return fail(c, ICX_ERR_INVALID, "null argument");
  if (!c->ready) return fail(c, ICX_ERR_INVALID, "icx_setup has not completed");
  const int D = icx::face_minb_default(c->phys.pde, c->phys.beta1 != 0.0);
  if (t->face_minb != 0 && (t->face_minb < D - 1 || t->face_minb > D + 1))
    return fail(c, ICX_ERR_INVALID, "face_minb: 0 or " + std::to_string(D - 1) + ".." + std::to_string(D + 1));
  bool vol_ok = t->vol_threads == 0 && t->vol_minb == 0;
  for (const icx::VolTile& v : icx::kVolTiles) vol_ok = vol_ok || (t->vol_threads == v.threads && t->vol_minb == v.minb);
  if (!vol_ok) return fail(c, ICX_ERR_INVALID, "vol_threads / vol_minb: not a compiled volume tile");
  const int bs = c->dm.nb * c->dm.neq;
  for (int k = 0; k < 2; ++k) {
    if (!icx::flow_rows_compiled(bs, t->ilu_rows[k]))
      return fail(c, ICX_ERR_INVALID, "ilu_rows: not compiled for this block size");
    if (t->ilu_ctas[k] < 0 || t->ilu_ctas[k] > MAX_CTAS) return fail(c, ICX_ERR_INVALID, "ilu_ctas: 0..4");
    if (t->ilu_sched[k] < 0 || t->ilu_sched[k] > 5) return fail(c, ICX_ERR_INVALID, "ilu_sched: 0..5");
    if (t->ilu_sched[k] >= 3 && t->ilu_ctas[k] > 3)
      return fail(c, ICX_ERR_INVALID, "ilu_ctas: 0..3 for the group applies (512 / 256 / 128 threads per CTA)");
  }
  TileChoice& d = c->dm.tile;
  d.face_minb = t->face_minb;
  d.vol_threads = t->vol_threads;
  d.vol_minb = t->vol_minb;
  for (int k = 0; k < 2; ++k) {
    d.flow_rows[k] = t->ilu_rows[k];
    d.flow_ctas[k] = t->ilu_ctas[k];
    d.flow_sched[k] = t->ilu_sched[k];
  }
  return ICX_OK;
}

icx_status icx_autotune(icx_ctx* c, const double* d_u, int parts, icx_tune_report* rep) {
  if (!c) return ICX_ERR_INVALID;
  if (!c->ready) return fail(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u) return fail(c, ICX_ERR_INVALID, "null state");
  if ((parts & TUNE_ALL) == 0 || (parts & ~(TUNE_ALL | ICX_TUNE_RETIME)) != 0)
    return fail(c, ICX_ERR_INVALID, "parts: a combination of ICX_TUNE_RESIDUAL, _ILU, _ILU_FP32 (| _RETIME)");
  TCK(cudaSetDevice(c->device));
  icx_tune_report local{};
  icx_tune_report* R = rep ? rep : &local;
  *R = icx_tune_report{};
  const Key key = key_of(c);
  CacheEntry cached;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) cached = it->second;
  }
  const bool retime = parts & ICX_TUNE_RETIME;
  int todo = parts & TUNE_ALL;
  icx::TileChoice& t = c->dm.tile;
  if (!retime) {
    const int hit = todo & cached.parts;
    if (hit & ICX_TUNE_RESIDUAL) {
      t.face_minb = cached.tile.face_minb;
      t.vol_threads = cached.tile.vol_threads;
      t.vol_minb = cached.tile.vol_minb;
    }
    for (int pi = 0; pi < 2; ++pi)
      if (hit & (pi == 0 ? ICX_TUNE_ILU : ICX_TUNE_ILU_FP32)) {
        t.flow_rows[pi] = cached.tile.flow_rows[pi];
        t.flow_ctas[pi] = cached.tile.flow_ctas[pi];
        t.flow_sched[pi] = cached.tile.flow_sched[pi];
      }
    R->from_cache = hit;
    todo &= ~hit;
  }
  icx_status st = ICX_OK;
  if (todo) {
    Tuner tu;
    tu.c = c;
    if ((st = tu.init()) != ICX_OK) return st;
    if (todo & ICX_TUNE_RESIDUAL) st = tu.residual(d_u, &R->residual_ms_default, &R->residual_ms_tuned);
    if (st == ICX_OK && (todo & (ICX_TUNE_ILU | ICX_TUNE_ILU_FP32)))
      st = tu.ilu(d_u, todo & ICX_TUNE_ILU, todo & ICX_TUNE_ILU_FP32, R->ilu_ms_default, R->ilu_ms_tuned);
    R->n_timed = tu.timed;
    R->n_rejected = tu.rejected;
    if (st != ICX_OK) return st;
    std::lock_guard<std::mutex> lk(g_mu);
    CacheEntry& ce = g_cache[key];
    if (todo & ICX_TUNE_RESIDUAL) {
      ce.tile.face_minb = t.face_minb;
      ce.tile.vol_threads = t.vol_threads;
      ce.tile.vol_minb = t.vol_minb;
    }
    for (int pi = 0; pi < 2; ++pi)
      if (todo & (pi == 0 ? ICX_TUNE_ILU : ICX_TUNE_ILU_FP32)) {
        ce.tile.flow_rows[pi] = t.flow_rows[pi];
        ce.tile.flow_ctas[pi] = t.flow_ctas[pi];
        ce.tile.flow_sched[pi] = t.flow_sched[pi];
      }
    ce.parts |= todo;
  }
  to_public(t, &R->chosen);
  return ICX_OK;
}

}  // extern "C"
