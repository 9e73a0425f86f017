// FD Jacobian, BSR linear algebra and the Newton driver (filled in below).
#include "icx_internal.h"

extern "C" {
icx_status icx_form_jacobian_fd(icx_ctx* c, const double*, double*, double*, double, void*) {
  if (c) c->err = "not built yet";
  return ICX_ERR_UNSUPPORTED;
}
icx_status icx_bsr_spmv(icx_ctx* c, const double*, const double*, double*, void*) {
  if (c) c->err = "not built yet";
  return ICX_ERR_UNSUPPORTED;
}
icx_status icx_newton_default_options(icx_newton_options*) { return ICX_ERR_UNSUPPORTED; }
icx_status icx_newton_solve(icx_ctx*, double*, const icx_newton_options*, icx_newton_report*) {
  return ICX_ERR_UNSUPPORTED;
}
}
