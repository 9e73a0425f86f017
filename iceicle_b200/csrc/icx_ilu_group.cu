// Launchers of the block-ILU(0) applies on element groups (tiles): one CTA
// per group, the register form (schedule 3), the shared-memory staged form
// (schedule 4) and the one-lane-per-row form (schedule 5), for every
// compiled block size, rows per task and CTA size. The kernels are in
// icx_blockrow.cuh.
#include <cuda_runtime.h>

#include "icx_internal.h"
#include "icx_linalg.h"
#include "icx_blockrow.cuh"

namespace icx {

namespace {

// threads per CTA of the group applies for a launch-shape choice k (the
// tile choice's CTAs-per-SM field): 0 the default, 1 / 2 / 3 512 / 256 / 128
template <class TA>
int group_threads_for(int k) {
  switch (k) {
    case 0: return group_threads<TA>();
    case 1: return 512;
    case 2: return 256;
    case 3: return 128;
    default: return 0;
  }
}

int smem_optin_bytes() {
  static int v = -1;
  if (v < 0) {
    int dev = 0, b = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&b, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      b = 0;
    v = b;
  }
  return v;
}

size_t smem_avail() {
  const size_t optin = (size_t)smem_optin_bytes();
  return optin > 2048 ? optin - 2048 : 0;  // less the kernels' static shared memory and a margin
}

struct GroupKernel {
  const void* kern;
  size_t smem;
};

template <int B, int R, class TA, int NT>
GroupKernel group_kernel_if_fit(bool staged, int gmax, int nlev_max) {
  if constexpr (flow_rows_fit(B, (B + 31) / 32, R)) {
    if (staged && nlev_max <= kGroupLevelsSmem) {
      // the deepest ring that fits beside the group's task-table entries
      const size_t info = (size_t)2 * gmax * sizeof(int4);
      const size_t ring = (size_t)(NT / 32) * group_slot_bytes<B, R, TA>();
      const size_t avail = smem_avail();
      if (info + 3 * ring <= avail) return {(const void*)ilu_apply_group_async_kernel<B, R, TA, NT, 3>, info + 3 * ring};
      if (info + 2 * ring <= avail) return {(const void*)ilu_apply_group_async_kernel<B, R, TA, NT, 2>, info + 2 * ring};
    }
    return {(const void*)ilu_apply_group_kernel<B, R, TA, NT>, 0};
  }
  return {nullptr, 0};
}

template <int B, int R, class TA>
GroupKernel group_kernel_nt(int nt, bool staged, int gmax, int nlev_max) {
  switch (nt) {
    case 128: return group_kernel_if_fit<B, R, TA, 128>(staged, gmax, nlev_max);
    case 256: return group_kernel_if_fit<B, R, TA, 256>(staged, gmax, nlev_max);
    case 512: return group_kernel_if_fit<B, R, TA, 512>(staged, gmax, nlev_max);
    default: return {nullptr, 0};
  }
}

// schedule 5: one lane per row, where the group's vectors fit
template <int B, class TA>
GroupKernel group_rows_kernel(int nt, int gmax, int nlev_max) {
  const size_t sm = group_rows_smem<typename ComputeOf<TA>::type>(gmax, B);
  if (nlev_max > kGroupLevelsSmem || sm > smem_avail()) return {nullptr, 0};
  switch (nt) {
    case 128: return {(const void*)ilu_apply_group_rows_kernel<B, TA, 128>, sm};
    case 256: return {(const void*)ilu_apply_group_rows_kernel<B, TA, 256>, sm};
    case 512: return {(const void*)ilu_apply_group_rows_kernel<B, TA, 512>, sm};
    default: return {nullptr, 0};
  }
}

template <int B, class TA>
GroupKernel group_kernel_for(int rows, int nt, bool staged, int gmax, int nlev_max) {
  switch (rows ? rows : FlowCfg<B>::R_DEFAULT) {
    case 2: return group_kernel_nt<B, 2, TA>(nt, staged, gmax, nlev_max);
    case 4: return group_kernel_nt<B, 4, TA>(nt, staged, gmax, nlev_max);
    case 6: return group_kernel_nt<B, 6, TA>(nt, staged, gmax, nlev_max);
    case 8: return group_kernel_nt<B, 8, TA>(nt, staged, gmax, nlev_max);
    default: return {nullptr, 0};
  }
}

template <class TA>
cudaError_t ilu_apply_groups_t(const DeviceMesh& dm, const IluGroupShape& gs, const int* task, const int* glev,
                               const int* glev_ptr, int rows, int ctas, const TA* LU, const TA* Uinv,
                               const double* x, double* y, double* f, int* err, cudaStream_t s) {
  if (gs.ngroups <= 0) return cudaErrorInvalidValue;
  const int bs = dm.nb * dm.neq;
  const int nt = group_threads_for<TA>(ctas);
  GroupKernel k{nullptr, 0};
#define ICX_ILUG_CASE(B)                                                                  \
  if (bs == B) {                                                                          \
    if (gs.sched == 5 && gs.loc) k = group_rows_kernel<B, TA>(nt, gs.gmax, gs.nlev_max);  \
    if (!k.kern) k = group_kernel_for<B, TA>(rows, nt, gs.sched >= 4, gs.gmax, gs.nlev_max); \
  }
  ICX_BLOCK_SIZES(ICX_ILUG_CASE)
#undef ICX_ILUG_CASE
  if (!k.kern) return cudaErrorInvalidValue;
  if (k.smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
    if (e != cudaSuccess) return e;
  }
  IluGroupArgs<TA> args{dm.E, dm.nnzb, LU, Uinv, x, f, y, err,
                        IluGroupPlan{gs.ngroups, reinterpret_cast<const int4*>(task), glev, glev_ptr, gs.gmax,
                                     reinterpret_cast<const int4*>(gs.loc)}};
  void* params[] = {&args};
  return cudaLaunchKernel(k.kern, dim3(gs.ngroups), dim3(nt), params, k.smem, s);
}

}  // namespace

cudaError_t la_ilu_apply_groups_bf16(const DeviceMesh& dm, const IluGroupShape& gs, const int* task,
                                     const int* glev, const int* glev_ptr, int ctas, const __nv_bfloat16* LU,
                                     const __nv_bfloat16* Uinv, const double* x, double* y, double* f, int* err,
                                     cudaStream_t s) {
  if (gs.ngroups <= 0 || !gs.loc) return cudaErrorInvalidValue;
  const int bs = dm.nb * dm.neq;
  const int nt = group_threads_for<float>(ctas);
  GroupKernel k{nullptr, 0};
#define ICX_ILUG16_CASE(B) \
  if (bs == B) k = group_rows_kernel<B, __nv_bfloat16>(nt, gs.gmax, gs.nlev_max);
  ICX_BLOCK_SIZES(ICX_ILUG16_CASE)
#undef ICX_ILUG16_CASE
  if (!k.kern) return cudaErrorNotSupported;  // the one-lane-per-row form does not fit
  if (k.smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
    if (e != cudaSuccess) return e;
  }
  IluGroupArgs<__nv_bfloat16> args{dm.E, dm.nnzb, LU, Uinv, x, f, y, err,
                                   IluGroupPlan{gs.ngroups, reinterpret_cast<const int4*>(task), glev, glev_ptr,
                                                gs.gmax, reinterpret_cast<const int4*>(gs.loc)}};
  void* params[] = {&args};
  return cudaLaunchKernel(k.kern, dim3(gs.ngroups), dim3(nt), params, k.smem, s);
}

bool group_rows_bf16_fits(const DeviceMesh& dm, const IluGroupShape& gs) {
  const int bs = dm.nb * dm.neq;
  const size_t sm = group_rows_smem<float>(gs.gmax, bs);
  return gs.loc && gs.nlev_max <= kGroupLevelsSmem && sm <= smem_avail();
}

cudaError_t la_ilu_apply_groups(const DeviceMesh& dm, const IluGroupShape& gs, const int* task, const int* glev,
                                const int* glev_ptr, int rows, int ctas, const double* LU, const double* Uinv,
                                const double* x, double* y, double* f, int* err, cudaStream_t s) {
  return ilu_apply_groups_t<double>(dm, gs, task, glev, glev_ptr, rows, ctas, LU, Uinv, x, y, f, err, s);
}

cudaError_t la_ilu_apply_groups_f32(const DeviceMesh& dm, const IluGroupShape& gs, const int* task,
                                    const int* glev, const int* glev_ptr, int rows, int ctas, const float* LU,
                                    const float* Uinv, const double* x, double* y, double* f, int* err,
                                    cudaStream_t s) {
  return ilu_apply_groups_t<float>(dm, gs, task, glev, glev_ptr, rows, ctas, LU, Uinv, x, y, f, err, s);
}

}  // namespace icx
