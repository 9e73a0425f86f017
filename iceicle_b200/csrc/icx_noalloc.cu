// Allocation-free residual entry point.
//
// icx_form_residual keeps its face-flux scratch in device memory that
// icx_setup allocates with cudaMalloc. Some callers cannot allocate device
// memory at the point where they evaluate residuals: a host framework that
// owns all device memory through its own pool and forbids other allocations
// during a solve, or a time-critical loop that must not pay the implicit
// device-wide synchronisation of cudaMalloc/cudaFree. For them this entry
// point runs the same kernels with the face-flux scratch taken from a
// file-scope __device__ array of fixed size instead of from the context.
//
// Limits and rules:
//   * capacity: ICX_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB) per device, held
//     by every GPU that loads the library until the process exits. A problem
//     needs n_faces * nq_face * neq doubles (plus n_faces * 4 * nq_face when
//     sigma_ic != 0 with Burgers); larger problems are rejected with
//     ICX_ERR_SIZE before any launch.
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress while that device is current, and caches it; make
//     that first call before any stream capture on the device.
//   * all calls on a device share the one array, which keeps the contents of
//     the last call. Every scratch entry a call reads is written earlier in
//     the same call, so nothing has to be cleared; but calls whose kernels
//     overlap on the GPU (different streams, no ordering between them) race
//     on the array and must be serialised by the caller.
#include <mutex>

#include "icx_internal.h"

#define ICX_NOALLOC_SCRATCH_DOUBLES (1 << 20)
#define ICX_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double icx_noalloc_scratch[ICX_NOALLOC_SCRATCH_DOUBLES];

namespace {
double* g_scratch_ptr[ICX_NOALLOC_MAX_DEVICES] = {};
std::mutex g_scratch_mu;

// device address of the scratch array on `device` (which must be current)
cudaError_t scratch_address(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, icx_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}
}  // namespace

extern "C" icx_status icx_form_residual_noalloc(icx_ctx* c, const double* d_u, double* d_res, void* stream) {
  if (!c || !c->ready) {
    if (c) c->err = "icx_setup has not completed";
    return ICX_ERR_INVALID;
  }
  if (!d_u || !d_res) {
    c->err = "null device pointer";
    return ICX_ERR_INVALID;
  }
  if (c->device < 0 || c->device >= ICX_NOALLOC_MAX_DEVICES) {
    c->err = "device index beyond the allocation-free path's device table";
    return ICX_ERR_SIZE;
  }
  const icx::DeviceMesh& dm = c->dm;
  size_t need_flux = (size_t)dm.F * dm.nqf * dm.neq;
  bool ic = c->phys.pde == ICX_PDE_BURGERS && c->phys.sigma_ic != 0.0;
  size_t need_grad = ic ? (size_t)dm.F * 2 * dm.nqf * 2 : 0;
  if (need_flux + need_grad > (size_t)ICX_NOALLOC_SCRATCH_DOUBLES) {
    c->err = "problem needs more face scratch than the allocation-free path's fixed " +
             std::to_string(ICX_NOALLOC_SCRATCH_DOUBLES) + " doubles (" +
             std::to_string(need_flux + need_grad) + " needed); use icx_form_residual";
    return ICX_ERR_SIZE;
  }
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e == cudaSuccess && cur != c->device) e = cudaSetDevice(c->device);
  double* base = nullptr;
  if (e == cudaSuccess) e = scratch_address(c->device, &base);
  if (e != cudaSuccess) {
    if (cur >= 0 && cur != c->device) cudaSetDevice(cur);  // leave the caller's device current
    c->err = std::string("scratch address lookup: ") + cudaGetErrorString(e);
    return ICX_ERR_CUDA;
  }
  icx::DeviceMesh view = dm;  // same tables, scratch redirected to the static array
  view.face_flux = base;
  view.face_grad = base + need_flux;
  e = icx::launch_residual(view, c->phys, d_u, d_res, (cudaStream_t)stream);
  if (cur >= 0 && cur != c->device) cudaSetDevice(cur);
  if (e != cudaSuccess) {
    c->err = std::string("residual kernels: ") + cudaGetErrorString(e);
    return ICX_ERR_CUDA;
  }
  return ICX_OK;
}
