/*
 * Point callbacks of the synthetic workloads for the oracle and the
 * reference CPU build (test infrastructure only): boundary data, sources and
 * initial states with the signature of orc_point_fn, x[2] -> out[neq].
 * The product library exports its own copies (icx_wl_*); the oracle side
 * uses these so that the checker and the reference arm of the benchmark
 * load nothing from the code under test.
 */
#include "oracle.h"
#include "orc_ns_mms.h"

/* user = {n, v_0 .. v_{n-1}}: out = v */
void orc_wl_constant(const double* x, double* out, void* user) {
  (void)x;
  const double* p = (const double*)user;
  int n = (int)p[0];
  for (int k = 0; k < n; ++k) out[k] = p[1 + k];
}

/* user = {amp} or NULL: out = amp sin(2 pi x) sin(2 pi y) */
void orc_wl_sine_product(const double* x, double* out, void* user) {
  const double* p = (const double*)user;
  double amp = p ? p[0] : 1.0;
  out[0] = amp * sin(2.0 * M_PI * x[0]) * sin(2.0 * M_PI * x[1]);
}

/* user = {x0, slope, u_left, u_right}: u_left where x < x0 + slope y */
void orc_wl_oblique_step(const double* x, double* out, void* user) {
  const double* p = (const double*)user;
  out[0] = (x[0] < p[0] + p[1] * x[1]) ? p[2] : p[3];
}

/* user = {gamma, Pr, mu, pinf, A, u0, v0}: manufactured Navier-Stokes state */
void orc_wl_ns_mms_state(const double* x, double* out, void* user) {
  orc_ns_mms_state_eval(x[0], x[1], (const double*)user, out);
}

/* same parameters: its source term s = -div F */
void orc_wl_ns_mms_source(const double* x, double* out, void* user) {
  orc_ns_mms_source_eval(x[0], x[1], (const double*)user, out);
}
