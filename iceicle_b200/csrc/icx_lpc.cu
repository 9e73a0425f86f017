// Learned block preconditioner (preconditioner 5 of the Newton solver).
//
// The preconditioner is the block-ILU(0) factorisation of the Jacobian J
// (exact triangular solves, or Jacobi sweeps), followed by a learned
// correction of every element block:
//
//   z = (I + C) y,  y = ILU(r),  C = blockdiag(C_e)
//
// C_e comes from a graph network over the elements with one message-passing
// step over the face neighbours:
//
//   h1_e = relu(W1 x_e + b1),           x_e = J_ee / |J_ee|_F   (bs x bs values)
//   m_e  = mean over the face neighbours n of e of h1_n         (the message)
//   h2_e = relu(W2 [h1_e ; m_e] + b2)
//   C_e  = W3 h2_e + b3                                          (bs x bs values)
//
// The neighbours are the off-diagonal blocks of the element's block row of
// the BSR pattern. Its weights are trained on the Jacobians and Krylov
// residuals r of the plain solver to minimise the mean over residual samples
// of |r - J z(r)|^2 / |r|^2; the output layer starts at zero, so the
// untrained model is the ILU preconditioner itself. All MLP products run on
// the tensor cores (tcgen05.mma, BF16 operands, FP32 accumulation in tensor
// memory, TMA operand loads; icx_gemm_tc.cuh) in the forward and backward
// passes, with Adam on FP32 master weights. The Newton residual, its norm
// and the line search stay FP64, so the preconditioner changes iteration
// counts but not the converged state; the solver falls back to block-ILU(0)
// for any step whose linear solve misses its tolerance.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "icx_internal.h"
#include "icx_linalg.h"
#include "icx_gemm_tc.cuh"
#include "icx_mlp.cuh"

using icx::bf16;

struct icx_lpc {
  int device = 0, bs = 0, hidden = 0, D = 0;
  size_t np = 0;
  size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
  float* p = nullptr;     // FP32 master parameters: W1 [H][D], b1, W2 [H][2H], b2, W3 [D][H], b3
  float* grad = nullptr;
  float* m = nullptr;     // Adam moments
  float* v = nullptr;
  bf16* W1b = nullptr;    // BF16 copies for the products
  bf16* W2b = nullptr;
  bf16* W3b = nullptr;
  bf16* W2tb = nullptr;   // transposes for the backward pass (W2^T: [2H][H])
  bf16* W3tb = nullptr;
  long long steps = 0;
  // the output layer (W3, b3) is all zero: C = 0, the preconditioner is its
  // base (set from host parameters; training clears it)
  bool zero_correction = false;
};

// per-context buffers of the learned preconditioner (grown on demand)
struct icx_lpc_work {
  int E = 0, D = 0, H = 0, B = 0;
  int Ep = 0;  // E rounded up to a multiple of 8: the row length of the transposed activations (zero padded)
  long long n = 0;
  bf16 *X = nullptr, *H2 = nullptr;  // forward activations: X [E][D], H2 [E][H]
  bf16* H1 = nullptr;                // [E][2H]: h1 in columns 0..H-1, the neighbour mean m in H..2H-1
  float* C = nullptr;                // [E][bs][bs] correction
  // training only
  float *dC = nullptr, *dH = nullptr, *dH1 = nullptr;  // dH [E][2H] (also [E][H]), dH1 [E][H]
  bf16 *dCb = nullptr, *dCbT = nullptr, *XT = nullptr, *H1T = nullptr, *H2T = nullptr;  // H1T [2H][Ep]
  bf16 *dHb = nullptr, *dHT = nullptr;
  int* tpos = nullptr;      // position of the mirrored block (k, e) of each block (e, k)
  double *ys = nullptr, *as = nullptr, *t1 = nullptr, *t2 = nullptr, *rv = nullptr;
  double* dh = nullptr;
};

namespace {

using namespace icx;

int grid_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 148 * 64 ? (b < 1 ? 1 : b) : 148 * 64);
}

// C = A . B^T on the tensor cores (tcgen05, icx_gemm_tc.cuh)
cudaError_t gemm(int M, int N, int K, const bf16* A, int lda, const bf16* B, int ldb, const float* bias, bool relu,
                 float* C32, int ldc, bf16* C16, int ldc16, bool accumulate, int splits, cudaStream_t s) {
  return icx::gemm_tc(M, N, K, A, lda, B, ldb, bias, relu, C32, ldc, C16, ldc16, accumulate, splits, s);
}

// out (cols x ldo, ldo >= rows) = in^T; columns rows..ldo-1 of out are left as they are
cudaError_t transpose(int rows, int cols, const bf16* in, bf16* out, int ldo, cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_bf16_kernel<<<grid, block, 0, s>>>(rows, cols, in, out, ldo);
  return cudaGetLastError();
}

// X[e] = J_ee / |J_ee|_F in BF16 (zero block -> zeros)
__global__ void features_kernel(int E, int bs, const double* __restrict__ vals, const int* __restrict__ diag,
                                bf16* __restrict__ X) {
  const int e = blockIdx.x;
  if (e >= E) return;
  const int D = bs * bs;
  const double* b = vals + (size_t)diag[e] * D;
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < D; i += blockDim.x) s += b[i] * b[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  const double inv = red[0] > 0.0 ? 1.0 / sqrt(red[0]) : 0.0;
  for (int i = threadIdx.x; i < D; i += blockDim.x) X[(size_t)e * D + i] = __float2bfloat16_rn((float)(b[i] * inv));
}

// the message: H1[e][H + j] = mean over the face neighbours n of e of
// H1[n][j] (zero for an element without neighbours), FP32 sums of the BF16
// features in the pattern's column order
__global__ void message_mean_kernel(int E, int H, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                    bf16* __restrict__ H1) {
  const int e = blockIdx.x;
  if (e >= E) return;
  const int rb = rowptr[e], re = rowptr[e + 1];
  int deg = 0;
  for (int kb = rb; kb < re; ++kb) deg += colidx[kb] != e;
  const float inv = deg > 0 ? 1.f / (float)deg : 0.f;
  for (int j = threadIdx.x; j < H; j += blockDim.x) {
    float s = 0.f;
    for (int kb = rb; kb < re; ++kb) {
      const int n = colidx[kb];
      if (n != e) s += __bfloat162float(H1[(size_t)n * 2 * H + j]);
    }
    H1[(size_t)e * 2 * H + H + j] = __float2bfloat16_rn(s * inv);
  }
}

// backward of the message and of the first ReLU: with dcat = dLoss/d[h1 ; m]
// ([E][2H]), dh1_e = dcat_e[0..H) + sum over the neighbours n of e of
// dcat_n[H..2H) / deg(n) (the pattern is symmetric, so n's message reads e),
// then masked by h1_e > 0; FP32 and BF16 copies
__global__ void message_back_kernel(int E, int H, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                    const float* __restrict__ dcat, const bf16* __restrict__ H1,
                                    float* __restrict__ dH1, bf16* __restrict__ dH1b) {
  const int e = blockIdx.x;
  if (e >= E) return;
  for (int j = threadIdx.x; j < H; j += blockDim.x) {
    float s = dcat[(size_t)e * 2 * H + j];
    for (int kb = rowptr[e]; kb < rowptr[e + 1]; ++kb) {
      const int n = colidx[kb];
      if (n == e) continue;
      int deg = 0;
      for (int t = rowptr[n]; t < rowptr[n + 1]; ++t) deg += colidx[t] != n;
      s += dcat[(size_t)n * 2 * H + H + j] / (float)deg;
    }
    const float x = __bfloat162float(H1[(size_t)e * 2 * H + j]) > 0.f ? s : 0.f;
    dH1[(size_t)e * H + j] = x;
    dH1b[(size_t)e * H + j] = __float2bfloat16_rn(x);
  }
}

// out_e = sum over the blocks (e, k) of J_ke^T a_k (the mirrored block (k, e)
// sits at tpos[kb]); J in FP32, vectors FP64
__global__ void jt_kernel(int E, int bs, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                          const int* __restrict__ tpos, const float* __restrict__ J, const double* __restrict__ a,
                          double* __restrict__ out) {
  const int e = blockIdx.x, r = threadIdx.x;
  if (e >= E || r >= bs) return;
  double s = 0.0;
  for (int kb = rowptr[e]; kb < rowptr[e + 1]; ++kb) {
    const int k = colidx[kb];
    const float* Bk = J + (size_t)tpos[kb] * bs * bs;
    const double* ak = a + (size_t)k * bs;
    for (int c = 0; c < bs; ++c) s += (double)Bk[(size_t)c * bs + r] * ak[c];
  }
  out[(size_t)e * bs + r] = s;
}

// seeded standard normal vector (splitmix64 counter hash, Box-Muller)
__device__ inline unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void randn_kernel(long long n, unsigned long long seed, double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long a = mix64(seed ^ (2 * (unsigned long long)i)), b = mix64(seed ^ (2 * (unsigned long long)i + 1));
    const double u1 = ((a >> 11) + 1.0) * (1.0 / 9007199254740993.0);  // (0, 1]
    const double u2 = (b >> 11) * (1.0 / 9007199254740992.0);
    out[i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

// dC[e][i][j] = scale * sum_b a_b[e][i] * y_b[e][j]
__global__ void outer_kernel(int E, int bs, int B, long long n, const double* __restrict__ a,
                             const double* __restrict__ y, double scale, float* __restrict__ dC) {
  const long long tot = (long long)E * bs * bs;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const int D = bs * bs;
    const long long e = idx / D;
    const int ij = (int)(idx - e * D), i = ij / bs, j = ij - i * bs;
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += a[(size_t)b * n + e * bs + i] * y[(size_t)b * n + e * bs + j];
    dC[idx] = (float)(scale * s);
  }
}

// out[c] += sum over rows of M[r][c] (FP32), rows split over blockIdx.y
__global__ void colsum_kernel(int rows, int cols, const float* __restrict__ M, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const int chunk = (rows + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * chunk, r1 = min(rows, r0 + chunk);
  float s = 0.f;
  for (int r = r0; r < r1; ++r) s += M[(size_t)r * cols + c];
  atomicAdd(out + c, s);
}

// d <- d * (h > 0) in FP32, and its BF16 copy
__global__ void relu_back_kernel(long long n, float* __restrict__ d, const bf16* __restrict__ h, bf16* __restrict__ db) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = __bfloat162float(h[i]) > 0.f ? d[i] : 0.f;
    d[i] = x;
    db[i] = __float2bfloat16_rn(x);
  }
}

__global__ void to_bf16_kernel(long long n, const float* __restrict__ x, bf16* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// BF16 copy of a rows x cols FP32 matrix and of its transpose
__global__ void weights_bf16_kernel(int rows, int cols, const float* __restrict__ W, bf16* __restrict__ Wb,
                                    bf16* __restrict__ Wtb) {
  const long long n = (long long)rows * cols;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
    const bf16 b = __float2bfloat16_rn(W[i]);
    Wb[i] = b;
    if (Wtb) Wtb[(size_t)c * rows + r] = b;
  }
}

__global__ void adam_kernel(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

cudaError_t refresh_bf16(icx_lpc* L, cudaStream_t s) {
  const int H = L->hidden, D = L->D;
  weights_bf16_kernel<<<grid_for((long long)H * D), 256, 0, s>>>(H, D, L->p + L->oW1, L->W1b, nullptr);
  weights_bf16_kernel<<<grid_for((long long)H * 2 * H), 256, 0, s>>>(H, 2 * H, L->p + L->oW2, L->W2b, L->W2tb);
  weights_bf16_kernel<<<grid_for((long long)D * H), 256, 0, s>>>(D, H, L->p + L->oW3, L->W3b, L->W3tb);
  return cudaGetLastError();
}

template <class T>
cudaError_t grow(T*& p, size_t count) {
  if (p) cudaFree(p);
  p = nullptr;
  return cudaMalloc((void**)&p, sizeof(T) * (count ? count : 1));
}

icx_status fail(icx_ctx* c, icx_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

// inference buffers for E elements
cudaError_t ensure_infer(icx_ctx* c, const icx_lpc* L) {
  icx_lpc_work*& w = c->lpcw;
  const int E = c->dm.E;
  if (w && w->E == E && w->D == L->D && w->H == L->hidden) return cudaSuccess;
  icx::free_lpc_work(c);
  w = new icx_lpc_work();
  w->E = E;
  w->D = L->D;
  w->H = L->hidden;
  w->n = (long long)E * L->bs;
  cudaError_t e = grow(w->X, (size_t)E * L->D);
  if (e == cudaSuccess) e = grow(w->H1, (size_t)E * 2 * L->hidden);
  if (e == cudaSuccess) e = grow(w->H2, (size_t)E * L->hidden);
  if (e == cudaSuccess) e = grow(w->C, (size_t)E * L->D);
  return e;
}

cudaError_t ensure_train(icx_ctx* c, const icx_lpc* L, int B) {
  icx_lpc_work* w = c->lpcw;
  if (w->dC && w->B >= B) return cudaSuccess;
  const size_t E = w->E, D = L->D, H = L->hidden;
  w->B = B;
  w->Ep = (w->E + 7) / 8 * 8;
  const size_t Ep = w->Ep;
  cudaError_t e = grow(w->dC, E * D);
  if (e == cudaSuccess) e = grow(w->dCb, E * D);
  if (e == cudaSuccess) e = grow(w->dCbT, Ep * D);
  if (e == cudaSuccess) e = grow(w->XT, Ep * D);
  if (e == cudaSuccess) e = grow(w->H1T, Ep * 2 * H);
  if (e == cudaSuccess) e = grow(w->H2T, Ep * H);
  if (e == cudaSuccess) e = grow(w->dH, E * 2 * H);
  if (e == cudaSuccess) e = grow(w->dH1, E * H);
  if (e == cudaSuccess) e = grow(w->dHb, E * H);
  if (e == cudaSuccess) e = grow(w->dHT, Ep * H);
  // the padding columns of the transposes stay zero
  bf16* zp[] = {w->dCbT, w->XT, w->H1T, w->H2T, w->dHT};
  size_t zn[] = {Ep * D, Ep * D, Ep * 2 * H, Ep * H, Ep * H};
  for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaMemset(zp[i], 0, sizeof(bf16) * zn[i]);
  if (e == cudaSuccess) e = grow(w->ys, (size_t)B * w->n);
  if (e == cudaSuccess) e = grow(w->as, (size_t)B * w->n);
  if (e == cudaSuccess) e = grow(w->t1, (size_t)w->n);
  if (e == cudaSuccess) e = grow(w->t2, (size_t)w->n);
  if (e == cudaSuccess) e = grow(w->rv, (size_t)w->n);
  if (e == cudaSuccess) e = grow(w->dh, 4);
  if (e != cudaSuccess) return e;
  // mirrored block positions of the (symmetric) element pattern
  const DeviceMesh& dm = c->dm;
  std::vector<int> rp(dm.E + 1), ci(dm.nnzb), tp(dm.nnzb, -1);
  e = cudaMemcpy(rp.data(), dm.bsr_rowptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(ci.data(), dm.bsr_colidx, sizeof(int) * ci.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  for (int r = 0; r < dm.E; ++r)
    for (int kb = rp[r]; kb < rp[r + 1]; ++kb) {
      const int k = ci[kb];
      for (int kt = rp[k]; kt < rp[k + 1]; ++kt)
        if (ci[kt] == r) tp[kb] = kt;
      if (tp[kb] < 0) return cudaErrorInvalidValue;  // pattern not symmetric
    }
  e = grow(w->tpos, tp.size());
  if (e == cudaSuccess) e = cudaMemcpy(w->tpos, tp.data(), sizeof(int) * tp.size(), cudaMemcpyHostToDevice);
  return e;
}

// H1[:, :H] = relu(X W1^T + b1), H1[:, H:] = neighbour mean of H1[:, :H],
// H2 = relu(H1 W2^T + b2), C = H2 W3^T + b3; rowptr / colidx: the BSR pattern
cudaError_t mlp_forward(const icx_lpc* L, icx_lpc_work* w, const int* rowptr, const int* colidx, cudaStream_t s) {
  const int E = w->E, D = L->D, H = L->hidden;
  cudaError_t e = gemm(E, H, D, w->X, D, L->W1b, D, L->p + L->ob1, true, nullptr, 0, w->H1, 2 * H, false, 1, s);
  if (e != cudaSuccess) return e;
  message_mean_kernel<<<E, 128, 0, s>>>(E, H, rowptr, colidx, w->H1);
  e = gemm(E, H, 2 * H, w->H1, 2 * H, L->W2b, 2 * H, L->p + L->ob2, true, nullptr, 0, w->H2, H, false, 1, s);
  if (e == cudaSuccess) e = gemm(E, D, H, w->H2, H, L->W3b, H, L->p + L->ob3, false, w->C, D, nullptr, 0, false, 1, s);
  return e;
}

// gradients of the parameters (into L->grad, which the caller zeroed) from dC = dLoss/dC
cudaError_t mlp_backward(icx_lpc* L, icx_lpc_work* w, const int* rowptr, const int* colidx, cudaStream_t s) {
  const int E = w->E, D = L->D, H = L->hidden, Ep = w->Ep;
  const int split = 32;
  const long long ED = (long long)E * D, EH = (long long)E * H;
  cudaError_t e = cudaSuccess;
  to_bf16_kernel<<<grid_for(ED), 256, 0, s>>>(ED, w->dC, w->dCb);
  if ((e = transpose(E, D, w->dCb, w->dCbT, Ep, s)) != cudaSuccess) return e;
  if ((e = transpose(E, H, w->H2, w->H2T, Ep, s)) != cudaSuccess) return e;
  if ((e = transpose(E, 2 * H, w->H1, w->H1T, Ep, s)) != cudaSuccess) return e;
  // layer 3
  if ((e = gemm(D, H, Ep, w->dCbT, Ep, w->H2T, Ep, nullptr, false, L->grad + L->oW3, H, nullptr, 0, true, split, s)))
    return e;
  colsum_kernel<<<dim3((D + 255) / 256, 64), 256, 0, s>>>(E, D, w->dC, L->grad + L->ob3);
  if ((e = gemm(E, H, D, w->dCb, D, L->W3tb, D, nullptr, false, w->dH, H, nullptr, 0, false, 1, s))) return e;
  relu_back_kernel<<<grid_for(EH), 256, 0, s>>>(EH, w->dH, w->H2, w->dHb);
  // layer 2, over [h1 ; m]
  if ((e = transpose(E, H, w->dHb, w->dHT, Ep, s)) != cudaSuccess) return e;
  if ((e = gemm(H, 2 * H, Ep, w->dHT, Ep, w->H1T, Ep, nullptr, false, L->grad + L->oW2, 2 * H, nullptr, 0, true,
                split, s)))
    return e;
  colsum_kernel<<<dim3((H + 255) / 256, 64), 256, 0, s>>>(E, H, w->dH, L->grad + L->ob2);
  if ((e = gemm(E, 2 * H, H, w->dHb, H, L->W2tb, H, nullptr, false, w->dH, 2 * H, nullptr, 0, false, 1, s))) return e;
  // the message step and the first ReLU
  message_back_kernel<<<E, 128, 0, s>>>(E, H, rowptr, colidx, w->dH, w->H1, w->dH1, w->dHb);
  // layer 1
  if ((e = transpose(E, H, w->dHb, w->dHT, Ep, s)) != cudaSuccess) return e;
  if ((e = gemm(H, D, Ep, w->dHT, Ep, w->XT, Ep, nullptr, false, L->grad + L->oW1, D, nullptr, 0, true, split, s)))
    return e;
  colsum_kernel<<<dim3((H + 255) / 256, 64), 256, 0, s>>>(E, H, w->dH1, L->grad + L->ob1);
  (void)EH;
  return cudaGetLastError();
}

}  // namespace

namespace icx {

void free_lpc_work(icx_ctx* c) {
  icx_lpc_work* w = c->lpcw;
  if (!w) return;
  void* ptrs[] = {w->X,  w->H1,  w->H2,  w->C,   w->dC,   w->dH, w->dH1, w->dCb, w->dCbT, w->XT, w->H1T,
                  w->H2T, w->dHb, w->dHT, w->tpos, w->ys, w->as, w->t1,  w->t2,   w->rv, w->dh};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete w;
  c->lpcw = nullptr;
}

// after the Jacobian (FP64, w->vals of the solver) is formed: features and C
cudaError_t lpc_build(icx_ctx* c, const double* vals, cudaStream_t s) {
  const icx_lpc* L = c->lpc;
  if (!L) return cudaErrorInvalidValue;
  cudaError_t e = ensure_infer(c, L);
  if (e != cudaSuccess) return e;
  features_kernel<<<c->dm.E, 256, 0, s>>>(c->dm.E, L->bs, vals, c->dm.bsr_diag, c->lpcw->X);
  e = mlp_forward(L, c->lpcw, c->dm.bsr_rowptr, c->dm.bsr_colidx, s);
  if (e != cudaSuccess) return e;
  // a tensor-core tile that gave up on a wait leaves C incomplete: report it
  int flag = 0;
  e = icx::gemm_tc_status(&flag, s);
  return e != cudaSuccess ? e : (flag ? cudaErrorLaunchTimeout : cudaSuccess);
}

bool lpc_zero_correction(const icx_ctx* c) { return c->lpc && c->lpc->zero_correction; }

// z = (I + C) y
cudaError_t lpc_apply(icx_ctx* c, const double* y, double* z, cudaStream_t s) {
  if (!c->lpcw || !c->lpcw->C) return cudaErrorInvalidValue;
  return la_block_diag_correct_f32(c->dm.E, c->lpc->bs, c->lpcw->C, y, z, s);
}

}  // namespace icx

extern "C" {

icx_status icx_lpc_create(icx_lpc** out, int device, int block_size, int hidden, unsigned long long seed) {
  if (!out || block_size < 1 || block_size > 64 || hidden < 8 || hidden % 8) return ICX_ERR_INVALID;
  if ((block_size * block_size) % 8) return ICX_ERR_UNSUPPORTED;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return ICX_ERR_NO_DEVICE;
  icx_lpc* L = new icx_lpc();
  L->device = device;
  L->bs = block_size;
  L->hidden = hidden;
  L->D = block_size * block_size;
  const size_t D = L->D, H = hidden;
  L->oW1 = 0;
  L->ob1 = L->oW1 + H * D;
  L->oW2 = L->ob1 + H;
  L->ob2 = L->oW2 + H * 2 * H;
  L->oW3 = L->ob2 + H;
  L->ob3 = L->oW3 + D * H;
  L->np = L->ob3 + D;
  // He-uniform hidden layers, zero output layer (C = 0: the untrained model is ILU_s)
  std::vector<float> h(L->np, 0.f);
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  const float a1 = std::sqrt(6.f / (float)D), a2 = std::sqrt(6.f / (float)(2 * H));
  for (size_t i = 0; i < H * D; ++i) h[L->oW1 + i] = a1 * u(rng);
  for (size_t i = 0; i < H * 2 * H; ++i) h[L->oW2 + i] = a2 * u(rng);
  cudaError_t e = cudaSuccess;
  float** fp[] = {&L->p, &L->grad, &L->m, &L->v};
  for (float** q : fp)
    if (e == cudaSuccess) e = cudaMalloc((void**)q, sizeof(float) * L->np);
  if (e == cudaSuccess) e = cudaMalloc((void**)&L->W1b, sizeof(bf16) * H * D);
  if (e == cudaSuccess) e = cudaMalloc((void**)&L->W2b, sizeof(bf16) * H * 2 * H);
  if (e == cudaSuccess) e = cudaMalloc((void**)&L->W3b, sizeof(bf16) * D * H);
  if (e == cudaSuccess) e = cudaMalloc((void**)&L->W2tb, sizeof(bf16) * H * 2 * H);
  if (e == cudaSuccess) e = cudaMalloc((void**)&L->W3tb, sizeof(bf16) * D * H);
  if (e == cudaSuccess) e = cudaMemcpy(L->p, h.data(), sizeof(float) * L->np, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(L->m, 0, sizeof(float) * L->np);
  if (e == cudaSuccess) e = cudaMemset(L->v, 0, sizeof(float) * L->np);
  if (e == cudaSuccess) e = refresh_bf16(L, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    icx_lpc_destroy(L);
    return ICX_ERR_CUDA;
  }
  *out = L;
  return ICX_OK;
}

void icx_lpc_destroy(icx_lpc* L) {
  if (!L) return;
  cudaSetDevice(L->device);
  void* ptrs[] = {L->p, L->grad, L->m, L->v, L->W1b, L->W2b, L->W3b, L->W2tb, L->W3tb};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete L;
}

icx_status icx_lpc_info(const icx_lpc* L, int* block_size, int* hidden, long long* n_params, long long* steps) {
  if (!L) return ICX_ERR_INVALID;
  if (block_size) *block_size = L->bs;
  if (hidden) *hidden = L->hidden;
  if (n_params) *n_params = (long long)L->np;
  if (steps) *steps = L->steps;
  return ICX_OK;
}

icx_status icx_lpc_get_params(const icx_lpc* L, float* host) {
  if (!L || !host) return ICX_ERR_INVALID;
  cudaSetDevice(L->device);
  return cudaMemcpy(host, L->p, sizeof(float) * L->np, cudaMemcpyDeviceToHost) == cudaSuccess ? ICX_OK : ICX_ERR_CUDA;
}

icx_status icx_lpc_set_params(icx_lpc* L, const float* host) {
  if (!L || !host) return ICX_ERR_INVALID;
  cudaSetDevice(L->device);
  if (cudaMemcpy(L->p, host, sizeof(float) * L->np, cudaMemcpyHostToDevice) != cudaSuccess) return ICX_ERR_CUDA;
  if (refresh_bf16(L, 0) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return ICX_ERR_CUDA;
  L->zero_correction = true;
  for (size_t i = L->oW3; i < L->np && L->zero_correction; ++i) L->zero_correction = host[i] == 0.0f;
  return ICX_OK;
}

icx_status icx_lpc_attach(icx_ctx* c, icx_lpc* L) {
  if (!c || !c->ready) return ICX_ERR_INVALID;
  if (L && (L->bs != c->dm.nb * c->dm.neq || L->device != c->device))
    return fail(c, ICX_ERR_INVALID, "model block size or device differs from the context's");
  c->lpc = L;
  if (!L) icx::free_lpc_work(c);
  return ICX_OK;
}

icx_status icx_lpc_forward(icx_ctx* c, const double* d_vals, float* d_corr) {
  if (!c || !c->ready || !c->lpc || !d_vals) return fail(c, ICX_ERR_INVALID, "no model attached");
  cudaSetDevice(c->device);
  cudaError_t e = icx::lpc_build(c, d_vals, 0);
  if (e == cudaSuccess && d_corr)
    e = cudaMemcpyAsync(d_corr, c->lpcw->C, sizeof(float) * (size_t)c->dm.E * c->lpc->D, cudaMemcpyDeviceToDevice, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  return e == cudaSuccess ? ICX_OK : fail(c, ICX_ERR_CUDA, std::string("lpc forward: ") + cudaGetErrorString(e));
}

icx_status icx_lpc_train(icx_ctx* c, const double* d_vals, int n_samples, const double* d_samples,
                         const icx_lpc_train_options* o, icx_lpc_train_report* rep) {
  if (!c || !c->ready || !c->lpc || !d_vals || !d_samples || n_samples < 1 || !o)
    return fail(c, ICX_ERR_INVALID, "train: bad arguments or no model attached");
  if (o->batch < 1 || o->batch > 64 || o->steps < 0 || o->sweeps < 0 || o->sweeps > 16 || o->random < 0 ||
      o->random > o->batch)
    return fail(c, ICX_ERR_INVALID, "train: batch in 1..64, random in 0..batch, sweeps in 0..16");
  icx_lpc* L = c->lpc;
  cudaSetDevice(c->device);
  cudaStream_t s = 0;
  if (o->steps > 0) L->zero_correction = false;
  // the ILU(0) factors (FP32 copies) of this Jacobian, as preconditioner 5 applies them
  icx_status st = icx::solver_prepare_pc(c, d_vals, 4, o->sweeps);
  if (st != ICX_OK) return st;
  cudaError_t e = ensure_infer(c, L);
  if (e == cudaSuccess) e = ensure_train(c, L, o->batch);
  if (e != cudaSuccess) return fail(c, ICX_ERR_CUDA, std::string("train buffers: ") + cudaGetErrorString(e));
  icx_lpc_work* w = c->lpcw;
  const DeviceMesh& dm = c->dm;
  const long long n = w->n;
  const float* J32 = icx::solver_vals32(c);
  features_kernel<<<dm.E, 256, 0, s>>>(dm.E, L->bs, d_vals, dm.bsr_diag, w->X);
  if ((e = transpose(dm.E, L->D, w->X, w->XT, w->Ep, s)) != cudaSuccess) return fail(c, ICX_ERR_CUDA, "transpose");
  std::mt19937_64 rng(o->seed ^ (0x9e3779b97f4a7c15ull * (unsigned long long)(L->steps + 1)));
  std::vector<double> hnorm(2 * o->batch);
  double first = 0.0, last = 0.0;
  for (int it = 0; it < o->steps; ++it) {
    if ((e = mlp_forward(L, w, dm.bsr_rowptr, dm.bsr_colidx, s)) != cudaSuccess) break;
    // residual after the preconditioner, for each sample b: g = r - J (I + C) ILU_s(r)
    double loss = 0.0;
    for (int b = 0; b < o->batch && e == cudaSuccess; ++b) {
      const double* r = d_samples + (size_t)(rng() % (unsigned long long)n_samples) * n;
      if (b < o->random) {
        randn_kernel<<<grid_for(n), 256, 0, s>>>(n, rng(), w->rv);
        r = w->rv;
      }
      double* y = w->ys + (size_t)b * n;
      double* a = w->as + (size_t)b * n;
      e = icx::solver_apply_pc(c, o->sweeps > 0 ? 4 : 2, true, r, y, s);
      if (e == cudaSuccess) e = icx::lpc_apply(c, y, w->t1, s);
      if (e == cudaSuccess) e = icx::launch_bsr_spmv_f32(dm, J32, w->t1, w->t2, s);
      if (e == cudaSuccess) e = icx::la_xpay(n, r, -1.0, w->t2, w->t2, s);  // g
      if (e == cudaSuccess) e = icx::la_dot_to(n, r, r, w->dh, s);
      if (e == cudaSuccess) e = icx::la_dot_to(n, w->t2, w->t2, w->dh + 1, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(&hnorm[2 * b], w->dh, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) break;
      const double rr = hnorm[2 * b] > 0.0 ? hnorm[2 * b] : 1.0;
      loss += hnorm[2 * b + 1] / rr;
      jt_kernel<<<dm.E, 64, 0, s>>>(dm.E, L->bs, dm.bsr_rowptr, dm.bsr_colidx, w->tpos, J32, w->t2, a);
      e = icx::la_axpby(n, 0.0, a, -2.0 / rr, a, s);  // a = -2 J^T g / |r|^2
    }
    if (e != cudaSuccess) break;
    loss /= o->batch;
    if (it == 0) first = loss;
    last = loss;
    if (rep && it < 64) rep->loss_history[it] = loss;
    outer_kernel<<<grid_for((long long)dm.E * L->D), 256, 0, s>>>(dm.E, L->bs, o->batch, n, w->as, w->ys,
                                                                  1.0 / o->batch, w->dC);
    if ((e = cudaMemsetAsync(L->grad, 0, sizeof(float) * L->np, s)) != cudaSuccess) break;
    if ((e = mlp_backward(L, w, dm.bsr_rowptr, dm.bsr_colidx, s)) != cudaSuccess) break;
    ++L->steps;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)L->steps), c2 = 1.f - std::pow(b2, (float)L->steps);
    adam_kernel<<<grid_for((long long)L->np), 256, 0, s>>>((long long)L->np, L->p, L->grad, L->m, L->v,
                                                           (float)o->lr, b1, b2, 1e-8f, c1, c2);
    if ((e = refresh_bf16(L, s)) != cudaSuccess) break;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    int flag = 0;
    e = icx::gemm_tc_status(&flag, s);
    if (e == cudaSuccess && flag) e = cudaErrorLaunchTimeout;
  }
  if (e != cudaSuccess) return fail(c, ICX_ERR_CUDA, std::string("train: ") + cudaGetErrorString(e));
  if (rep) {
    rep->steps = o->steps;
    rep->loss_first = first;
    rep->loss_last = last;
  }
  return ICX_OK;
}

icx_status icx_lpc_calibrate(icx_ctx* c, const double* d_vals, int n_samples, const double* d_samples, int sweeps,
                             double sums[3]) {
  if (!c || !c->ready || !c->lpc || !d_vals || !d_samples || n_samples < 1 || !sums || sweeps < 0 || sweeps > 16)
    return fail(c, ICX_ERR_INVALID, "calibrate: bad arguments or no model attached");
  icx_lpc* L = c->lpc;
  cudaSetDevice(c->device);
  cudaStream_t s = 0;
  icx_status st = icx::solver_prepare_pc(c, d_vals, 4, sweeps);
  if (st != ICX_OK) return st;
  cudaError_t e = ensure_infer(c, L);
  if (e == cudaSuccess) e = ensure_train(c, L, 1);
  if (e == cudaSuccess) e = icx::lpc_build(c, d_vals, s);
  if (e != cudaSuccess) return fail(c, ICX_ERR_CUDA, std::string("calibrate: ") + cudaGetErrorString(e));
  icx_lpc_work* w = c->lpcw;
  const long long n = w->n;
  const float* J32 = icx::solver_vals32(c);
  const DeviceMesh& dm = c->dm;
  sums[0] = sums[1] = sums[2] = 0.0;
  double h[4];
  for (int k = 0; k < n_samples && e == cudaSuccess; ++k) {
    // a = r - J y (the base preconditioner's residual), b = J C y (the
    // correction's change to it): |r - J (I + g C) y|^2 = |a - g b|^2
    const double* r = d_samples + (size_t)k * n;
    double* y = w->ys;
    double* a = w->as;
    e = icx::solver_apply_pc(c, sweeps > 0 ? 4 : 2, true, r, y, s);
    if (e == cudaSuccess) e = icx::launch_bsr_spmv_f32(dm, J32, y, w->t2, s);
    if (e == cudaSuccess) e = icx::la_xpay(n, r, -1.0, w->t2, a, s);
    if (e == cudaSuccess) e = icx::lpc_apply(c, y, w->t1, s);
    if (e == cudaSuccess) e = icx::la_xpay(n, w->t1, -1.0, y, w->t1, s);  // C y
    if (e == cudaSuccess) e = icx::launch_bsr_spmv_f32(dm, J32, w->t1, w->t2, s);
    if (e == cudaSuccess) e = icx::la_dot_to(n, r, r, w->dh, s);
    if (e == cudaSuccess) e = icx::la_dot_to(n, a, w->t2, w->dh + 1, s);
    if (e == cudaSuccess) e = icx::la_dot_to(n, w->t2, w->t2, w->dh + 2, s);
    if (e == cudaSuccess) e = icx::la_dot_to(n, a, a, w->dh + 3, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, w->dh, 4 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) break;
    const double rr = h[0] > 0.0 ? h[0] : 1.0;
    sums[0] += h[1] / rr;
    sums[1] += h[2] / rr;
    sums[2] += h[3] / rr;
  }
  if (e != cudaSuccess) return fail(c, ICX_ERR_CUDA, std::string("calibrate: ") + cudaGetErrorString(e));
  return ICX_OK;
}

}  // extern "C"
