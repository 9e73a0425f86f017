// Residuals of a sequence of states held in host memory: the copy of state
// k + 1 to the device, the residual kernels of state k and the copy of
// residual k - 1 back to the host run at the same time, on three streams
// (host-to-device copy engine, SMs, device-to-host copy engine) with two
// device buffer pairs used in turn. Events order the three stages of a state
// and keep a buffer from being overwritten before its previous user is done;
// the residual kernels of consecutive states stay ordered, because they share
// the context's face scratch.
#include <string>

#include "icx_internal.h"

struct icx_host_pipe {
  long long n = 0;
  int device = 0;
  cudaStream_t s_in = nullptr, s_run = nullptr, s_out = nullptr;
  double* d_u[2] = {nullptr, nullptr};
  double* d_r[2] = {nullptr, nullptr};
  cudaEvent_t copied_in[2] = {nullptr, nullptr};   // d_u[b] holds its state
  cudaEvent_t computed[2] = {nullptr, nullptr};    // d_r[b] holds its residual, d_u[b] is free
  cudaEvent_t copied_out[2] = {nullptr, nullptr};  // d_r[b] is free
  cudaEvent_t t0 = nullptr, t1 = nullptr;
};

namespace icx {

void free_host_pipe(icx_ctx* c) {
  icx_host_pipe* p = c->hp;
  if (!p) return;
  cudaSetDevice(p->device);
  for (int b = 0; b < 2; ++b) {
    if (p->d_u[b]) cudaFree(p->d_u[b]);
    if (p->d_r[b]) cudaFree(p->d_r[b]);
    cudaEvent_t* evs[] = {&p->copied_in[b], &p->computed[b], &p->copied_out[b]};
    for (cudaEvent_t* e : evs)
      if (*e) cudaEventDestroy(*e);
  }
  if (p->t0) cudaEventDestroy(p->t0);
  if (p->t1) cudaEventDestroy(p->t1);
  cudaStream_t ss[] = {p->s_in, p->s_run, p->s_out};
  for (cudaStream_t s : ss)
    if (s) cudaStreamDestroy(s);
  delete p;
  c->hp = nullptr;
}

}  // namespace icx

namespace {

icx_status pipe_fail(icx_ctx* c, icx_status st, const std::string& m) {
  c->err = m;
  return st;
}

icx_status ensure_pipe(icx_ctx* c, long long n) {
  if (c->hp && c->hp->n == n) return ICX_OK;
  icx::free_host_pipe(c);
  icx_host_pipe* p = new icx_host_pipe();
  c->hp = p;
  p->n = n;
  p->device = c->device;
  cudaError_t e = cudaSuccess;
  cudaStream_t* ss[] = {&p->s_in, &p->s_run, &p->s_out};
  for (cudaStream_t* s : ss)
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaMalloc((void**)&p->d_u[b], sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc((void**)&p->d_r[b], sizeof(double) * n);
    cudaEvent_t* evs[] = {&p->copied_in[b], &p->computed[b], &p->copied_out[b]};
    for (cudaEvent_t* ev : evs)
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreate(&p->t0);
  if (e == cudaSuccess) e = cudaEventCreate(&p->t1);
  if (e != cudaSuccess) {
    icx::free_host_pipe(c);
    return pipe_fail(c, ICX_ERR_NOMEM, std::string("pipeline buffers: ") + cudaGetErrorString(e));
  }
  return ICX_OK;
}

}  // namespace

extern "C" icx_status icx_form_residuals_host(icx_ctx* c, int n_states, const double* h_u, double* h_res,
                                              double* elapsed_ms) {
  if (!c || !c->ready) return ICX_ERR_INVALID;
  if (n_states < 0 || (n_states > 0 && (!h_u || !h_res))) return pipe_fail(c, ICX_ERR_INVALID, "bad arguments");
  const long long n = (long long)c->dm.E * c->dm.nb * c->dm.neq;
  cudaSetDevice(c->device);
  icx_status st = ensure_pipe(c, n);
  if (st != ICX_OK) return st;
  icx_host_pipe* p = c->hp;
  // work already queued on the legacy stream (e.g. the caller's set-up) comes first
  cudaError_t e = cudaStreamSynchronize(0);
  if (e == cudaSuccess) e = cudaEventRecord(p->t0, p->s_in);
  for (int k = 0; k < n_states && e == cudaSuccess; ++k) {
    const int b = k & 1;
    const size_t bytes = sizeof(double) * (size_t)n;
    // state k in: d_u[b] is free once the kernels of state k - 2 have run
    if (k >= 2) e = cudaStreamWaitEvent(p->s_in, p->computed[b], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->d_u[b], h_u + (size_t)k * n, bytes, cudaMemcpyHostToDevice, p->s_in);
    if (e == cudaSuccess) e = cudaEventRecord(p->copied_in[b], p->s_in);
    // residual k: its state is in, and d_r[b] has been copied out for state k - 2
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_run, p->copied_in[b], 0);
    if (e == cudaSuccess && k >= 2) e = cudaStreamWaitEvent(p->s_run, p->copied_out[b], 0);
    if (e == cudaSuccess) e = icx::launch_residual(c->dm, c->phys, p->d_u[b], p->d_r[b], p->s_run);
    if (e == cudaSuccess) e = cudaEventRecord(p->computed[b], p->s_run);
    // residual k out
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_out, p->computed[b], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_res + (size_t)k * n, p->d_r[b], bytes, cudaMemcpyDeviceToHost, p->s_out);
    if (e == cudaSuccess) e = cudaEventRecord(p->copied_out[b], p->s_out);
  }
  if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_out, p->t0, 0);
  if (e == cudaSuccess) e = cudaEventRecord(p->t1, p->s_out);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->s_out);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->s_in);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->s_run);
  if (e != cudaSuccess) return pipe_fail(c, ICX_ERR_CUDA, std::string("host residual pipeline: ") + cudaGetErrorString(e));
  if (elapsed_ms) {
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, p->t0, p->t1);
    *elapsed_ms = e == cudaSuccess ? (double)ms : -1.0;
  }
  return ICX_OK;
}
