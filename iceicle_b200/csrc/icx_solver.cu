// C ABI of the FD Jacobian and BSR products; the Newton driver.
#include <cfloat>
#include <cmath>

#include "icx_internal.h"

namespace {
icx_status set_err(icx_ctx* c, icx_status st, const std::string& m) {
  if (c) c->err = m;
  return st;
}
}  // namespace

extern "C" {

icx_status icx_form_jacobian_fd(icx_ctx* c, const double* d_u, double* d_res, double* d_vals, double eps,
                                void* stream) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_u || !d_res || !d_vals) return set_err(c, ICX_ERR_INVALID, "null device pointer");
  if (!(eps > 0.0)) eps = std::sqrt(DBL_EPSILON);
  cudaError_t e = icx::launch_jacobian_fd(c->dm, c->phys, d_u, d_res, d_vals, eps, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string("jacobian kernels: ") + cudaGetErrorString(e));
  return ICX_OK;
}

icx_status icx_bsr_spmv(icx_ctx* c, const double* d_vals, const double* d_x, double* d_y, void* stream) {
  if (!c || !c->ready) return set_err(c, ICX_ERR_INVALID, "icx_setup has not completed");
  if (!d_vals || !d_x || !d_y) return set_err(c, ICX_ERR_INVALID, "null device pointer");
  cudaError_t e = icx::launch_bsr_spmv(c->dm, d_vals, d_x, d_y, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_err(c, ICX_ERR_CUDA, std::string("spmv: ") + cudaGetErrorString(e));
  return ICX_OK;
}

icx_status icx_newton_default_options(icx_newton_options*) { return ICX_ERR_UNSUPPORTED; }
icx_status icx_newton_solve(icx_ctx*, double*, const icx_newton_options*, icx_newton_report*) {
  return ICX_ERR_UNSUPPORTED;
}
}
