// Point callbacks for the synthetic workloads (boundary data, sources and
// initial states), exported so that C, C++ and Python callers can hand them
// to icx_disc_dirichlet / icx_disc_neumann / icx_disc_source.
#include <cmath>

#include "../../include/iceicle_b200.h"
#include "icx_ns_mms.h"

extern "C" {

void icx_wl_constant(const double* x, double* out, void* user) {
  (void)x;
  const double* p = (const double*)user;
  int n = (int)p[0];
  for (int k = 0; k < n; ++k) out[k] = p[1 + k];
}

void icx_wl_sine_product(const double* x, double* out, void* user) {
  const double* p = (const double*)user;
  double amp = p ? p[0] : 1.0;
  out[0] = amp * std::sin(2.0 * M_PI * x[0]) * std::sin(2.0 * M_PI * x[1]);
}

void icx_wl_oblique_step(const double* x, double* out, void* user) {
  const double* p = (const double*)user;  // {x0, slope, u_left, u_right}
  out[0] = (x[0] < p[0] + p[1] * x[1]) ? p[2] : p[3];
}

void icx_wl_ns_mms_state(const double* x, double* out, void* user) {
  const double* p = (const double*)user;
  icx_ns_mms_state(x[0], x[1], p[0], p[1], p[2], p[3], p[4], p[5], p[6], out);
}

void icx_wl_ns_mms_source(const double* x, double* out, void* user) {
  const double* p = (const double*)user;
  icx_ns_mms_source(x[0], x[1], p[0], p[1], p[2], p[3], p[4], p[5], p[6], out);
}
}
