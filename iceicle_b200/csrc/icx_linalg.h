// Device linear algebra used by the Newton solver (icx_linalg.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

#include "icx_internal.h"

namespace icx {

// CTAs of the multi-dot's first stage (8 per SM: enough warps in flight to
// stream the basis at full bandwidth)
constexpr int kMdotBlocks = 148 * 8;

struct LinalgWork {
  double* partial = nullptr;  // [64 vectors][kMdotBlocks] partial dot products
};

// d_out[j] = V_j . x for j < nvec, V_j = V + j * ld (deterministic two-stage reduction)
cudaError_t la_mdot(LinalgWork& w, long long n, const double* V, long long ld, int nvec, const double* x,
                    double* d_out, cudaStream_t s);
// w += sign * sum_j d_h[j] V_j
cudaError_t la_maxpy(long long n, const double* V, long long ld, int nvec, const double* d_h, double sign, double* w,
                     cudaStream_t s);
// the same two with an FP32 basis V (products and sums in FP64)
// matrix-free Jacobian products with slot = {|v|^2, c} on the device and
// h = c / |v|: up = u + h v, then y = (rp - r0) / h
cudaError_t la_fd_perturb(long long n, const double* u, const double* v, const double* slot, double* up,
                          cudaStream_t s);
cudaError_t la_fd_diff(long long n, const double* rp, const double* r0, const double* slot, double* y,
                       cudaStream_t s);
cudaError_t la_mdot32(LinalgWork& w, long long n, const float* V, long long ld, int nvec, const double* x,
                      double* d_out, cudaStream_t s);
cudaError_t la_maxpy32(long long n, const float* V, long long ld, int nvec, const double* d_h, double sign, double* w,
                       cudaStream_t s);
cudaError_t la_axpby(long long n, double a, const double* x, double b, double* y, cudaStream_t s);
// y = a x (y is not read)
cudaError_t la_scale(long long n, double a, const double* x, double* y, cudaStream_t s);
cudaError_t la_xpay(long long n, const double* x, double a, const double* y, double* z, cudaStream_t s);
// dst[b] = inv(src[blk_index[b]]) for b < nblk (bs x bs blocks); *flag set on a singular block
cudaError_t la_block_invert(int nblk, int bs, const double* src, const int* blk_index, double* dst, int* flag,
                            cudaStream_t s);
// y = x0 + sign * (strictly lower (lower = true) or strictly upper block part of A) v
cudaError_t la_tri_rows(const DeviceMesh& dm, bool lower, const double* A, const double* v, const double* x0,
                        double sign, double* y, cudaStream_t s);
cudaError_t la_tri_rows_f32(const DeviceMesh& dm, bool lower, const float* A, const double* v, const double* x0,
                            double sign, double* y, cudaStream_t s);
cudaError_t la_block_diag_apply(int E, int bs, const double* D, const double* x, double* y, cudaStream_t s);
// z = y + D y, D block diagonal in FP32 (FP32 accumulation)
cudaError_t la_block_diag_correct_f32(int E, int bs, const float* D, const double* y, double* z, cudaStream_t s);
// *d_out = x . y (device scalar, overwritten)
cudaError_t la_dot_to(long long n, const double* x, const double* y, double* d_out, cudaStream_t s);
// block-ILU(0) on the element block pattern in natural order, scheduled by
// levels: order lists the elements by ascending level (the anti-diagonal
// i + j of the element in its grid), lvl_off[l]..lvl_off[l+1] the elements of
// level l; every strictly lower neighbour of an element lies on a lower level.
// LU holds a copy of the BSR values on entry; on exit its strictly lower
// blocks are L, its upper blocks inv(U_ee) U_ek and Uinv the inv(U_ee).
// *flag: 1 if a diagonal block was singular, 2 if an index was out of range.
cudaError_t la_ilu_factor(const DeviceMesh& dm, const int* order, const std::vector<int>& lvl_off, double* LU,
                          double* Uinv, int* flag, cudaStream_t s);
// y = (LU)^-1 x in one cooperative launch scheduled by data flow: f = n
// doubles of scratch, cnt_f / cnt_b = E device counters each (zero before the
// first apply, never reset afterwards), epoch = 1 for the first apply after
// zeroing and +1 per apply; *err (device) is set to 1 if a dependency wait
// timed out, 2 if an index was out of range
// block-ILU(0) apply pipelined by grid rows (one nx x ny structured grid in
// natural order); cudaErrorNotSupported when the ny rows cannot all be resident
cudaError_t la_ilu_apply_rows(const DeviceMesh& dm, int nx, int ny, const double* LU, const double* Uinv,
                              const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b, unsigned epoch,
                              int* err, cudaStream_t s);
cudaError_t la_ilu_apply_rows_f32(const DeviceMesh& dm, int nx, int ny, const float* LU, const float* Uinv,
                                  const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b,
                                  unsigned epoch, int* err, cudaStream_t s);
cudaError_t la_ilu_apply_flow(const DeviceMesh& dm, const int* order, const double* LU, const double* Uinv,
                              const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b, unsigned epoch,
                              int* err, cudaStream_t s);
// FP32 matrix variants (FP32 values, FP32 accumulation; vectors stay FP64)
cudaError_t la_ilu_apply_flow_f32(const DeviceMesh& dm, const int* order, const float* LU, const float* Uinv,
                                  const double* x, double* y, double* f, unsigned* cnt_f, unsigned* cnt_b,
                                  unsigned epoch, int* err, cudaStream_t s);
// the same apply on element groups (tiles) whose factors couple no two
// groups: one CTA per group, levels of the group in turn (no cross-CTA
// waits); task (4 ints per entry, 16-byte aligned) / glev / glev_ptr as
// IluGroupPlan (icx_blockrow.cuh); rows =
// rows per warp task (0: the default); *err = 2 on an index out of range
// the plan's shape: groups, elements of the largest group, most levels of
// a group, the schedule (3 registers, 4 matrix rows staged in shared memory,
// 5 one lane per row with the group's vectors in shared memory; 5 and 4 fall
// back to the next lower one where their shared memory does not fit) and
// the entries by position within the group (IluGroupPlan::loc)
struct IluGroupShape {
  int ngroups, gmax, nlev_max, sched;
  const int* loc;
};
// ctas: threads per CTA, 0 the default (256 FP64, 512 FP32), 1 / 2 / 3
// 512 / 256 / 128 (icx_ilu_group.cu)
cudaError_t la_ilu_apply_groups(const DeviceMesh& dm, const IluGroupShape& gs, const int* task, const int* glev,
                                const int* glev_ptr, int rows, int ctas, const double* LU, const double* Uinv,
                                const double* x, double* y, double* f, int* err, cudaStream_t s);
cudaError_t la_ilu_apply_groups_f32(const DeviceMesh& dm, const IluGroupShape& gs, const int* task,
                                    const int* glev, const int* glev_ptr, int rows, int ctas, const float* LU,
                                    const float* Uinv, const double* x, double* y, double* f, int* err,
                                    cudaStream_t s);
// the one-lane-per-row group apply (schedule 5) on BF16 factors (FP32
// arithmetic); cudaErrorNotSupported where its shared memory does not fit
// (group_rows_bf16_fits says beforehand)
cudaError_t la_ilu_apply_groups_bf16(const DeviceMesh& dm, const IluGroupShape& gs, const int* task,
                                     const int* glev, const int* glev_ptr, int ctas, const __nv_bfloat16* LU,
                                     const __nv_bfloat16* Uinv, const double* x, double* y, double* f, int* err,
                                     cudaStream_t s);
bool group_rows_bf16_fits(const DeviceMesh& dm, const IluGroupShape& gs);
// y = x rounded to BF16
cudaError_t la_d2bf(long long n, const double* x, __nv_bfloat16* y, cudaStream_t s);
cudaError_t la_block_diag_apply_f32(int E, int bs, const float* D, const double* x, double* y, cudaStream_t s);
cudaError_t la_d2f(long long n, const double* x, float* y, cudaStream_t s);
cudaError_t la_f2d(long long n, const float* x, double* y, cudaStream_t s);
// dst block b = src block map[b] for b < nblk (bs x bs FP64 blocks)
cudaError_t la_gather_blocks(int nblk, int bs, const double* src, const int* map, double* dst, cudaStream_t s);
}  // namespace icx

#include <functional>
#include <string>

namespace icx {
// CUDA graphs of the GMRES Arnoldi steps, one per step index j, kept by their
// owner across solves. A graph holds every pointer and launch shape of the
// step, so it stays valid while `key` (the owner's description of the
// operators) is unchanged.
struct ArnoldiGraphs {
  unsigned long long key = 0;
  int m = 0;
  std::vector<cudaGraphExec_t> exec;  // [m]; null: not captured yet
  std::vector<int> seen;              // [m] eager runs of step j under this key
  bool failed = false;                // a capture failed under this key: eager steps only
  cudaStream_t cap = nullptr;         // capture stream
  double* hp = nullptr;               // pinned host copies of the steps' reductions, 2 x 3 (m + 2) doubles:
                                      // step j writes half j % 2, so step j + 1 may run while the host reads j
  cudaEvent_t done[2] = {nullptr, nullptr};  // completion of the last step launched into each half
  // drops the graphs (the key changed)
  void reset();
  // drops everything (owner teardown)
  void release();
};

// device buffers of a restarted GMRES(m) on vectors of length n
struct KrylovBuffers {
  long long n = 0;
  int m = 0;
  double* V = nullptr;  // (m + 1) x n basis
  double* w = nullptr;
  double* z = nullptr;
  double* r = nullptr;
  double* dh = nullptr;  // >= 3 (m + 2) device doubles
  LinalgWork* lw = nullptr;
  // optional FP32 basis (mixed precision): (m + 1) x n floats in place of V,
  // with the inner products and updates accumulated in FP64; vt is one FP64
  // vector, the operator's input widened from the basis
  float* V32 = nullptr;
  double* vt = nullptr;
  // optional Krylov samples: the true residual at every restart and every
  // `sample_every`-th Arnoldi vector, copied into samples[count] while count < cap
  double* samples = nullptr;
  int sample_cap = 0, sample_every = 0, sample_count = 0;
  // stall test (0: off): stop when the residual after a restart cycle is above
  // 0.9 of the residual `stall_cycles` cycles earlier
  int stall_cycles = 0;
  // classical Gram-Schmidt passes per Arnoldi step: 2 (a second pass every
  // step) or 1 (PETSc's default GMRES orthogonalisation, refinement never)
  int cgs_passes = 2;
  // optional: replay the Arnoldi steps as CUDA graphs (graph_key != 0; the
  // operators then launch only on the stream they are given, with arguments
  // that do not change between calls). Not used while sampling.
  ArnoldiGraphs* graphs = nullptr;
  unsigned long long graph_key = 0;
  int graph_launches = 0;  // out: Arnoldi steps replayed from a graph
};
// y = op(x), launched on stream s
using LinOp = std::function<cudaError_t(const double* x, double* y, cudaStream_t s)>;
double la_norm(LinalgWork& lw, long long n, const double* x, double* d_scratch, cudaStream_t s);
// x = A^-1 b, right-preconditioned by M (null: none); classical Gram-Schmidt
// with one re-orthogonalisation, FP64 Hessenberg/Givens on the host
icx_status gmres_op(KrylovBuffers& kb, const LinOp& A, const LinOp* M, int maxit, double rtol, const double* b,
                    double* x, int* iters, double* relres, cudaStream_t s, std::string* err);
}  // namespace icx
