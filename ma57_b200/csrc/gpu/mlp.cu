// Learned static-pivot perturbation: a small multilayer perceptron that maps
// per-front statistics to log10 of the first-attempt delta of
// Mode::StaticRegularized (the reference escalates one global delta by a
// fixed growth factor on every failed inertia check, solver.hpp:328-417).
//
// Network: x (kIn features, standardised) -> tanh(W1 x + b1) (kH) ->
// tanh(W2 h1 + b2) (kH) -> w3 . h2 + b3 (one output). FP64 throughout, so the
// gradients can be compared with a CPU restatement to rounding level.
//
// Kernels (one thread per sample; the network is tiny, the batch is the
// fronts of many factorizations):
//   mlp_forward_kernel   predictions, and the hidden activations for training
//   mlp_deltas_kernel    per sample: activations and back-propagated deltas
//   mlp_wgrad_kernel     per parameter and sample chunk: the gradient sum
//   mlp_reduce_kernel    sums the chunks in order (training is deterministic)
//   mlp_adam_kernel      Adam step on the parameter vector
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <algorithm>
#include <string>
#include <vector>

#include "../../../include/symla_gpu.h"
#include "context.hpp"

namespace {

constexpr int kIn = SYMLA_MLP_INPUTS;
constexpr int kH = SYMLA_MLP_HIDDEN;
// parameter vector layout
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * kIn;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH;
constexpr int kParams = kOffB3 + 1;
constexpr int kThreads = 128;

static_assert(kParams == SYMLA_MLP_PARAMS, "parameter count");

__device__ __forceinline__ void forward_one(const double* __restrict__ p, const double* __restrict__ x, double* h1,
                                            double* h2, double& y) {
  for (int j = 0; j < kH; ++j) {
    double a = p[kOffB1 + j];
    for (int i = 0; i < kIn; ++i) a = fma(p[kOffW1 + j * kIn + i], x[i], a);
    h1[j] = tanh(a);
  }
  for (int j = 0; j < kH; ++j) {
    double a = p[kOffB2 + j];
    for (int i = 0; i < kH; ++i) a = fma(p[kOffW2 + j * kH + i], h1[i], a);
    h2[j] = tanh(a);
  }
  double o = p[kOffB3];
  for (int i = 0; i < kH; ++i) o = fma(p[kOffW3 + i], h2[i], o);
  y = o;
}

__global__ void __launch_bounds__(kThreads) mlp_forward_kernel(const double* __restrict__ p,
                                                               const double* __restrict__ X, int B,
                                                               double* __restrict__ Y) {
  __shared__ double sp[kParams];
  for (int t = threadIdx.x; t < kParams; t += kThreads) sp[t] = p[t];
  __syncthreads();
  const int s = blockIdx.x * kThreads + threadIdx.x;
  if (s >= B) return;
  double x[kIn], h1[kH], h2[kH], y;
  for (int i = 0; i < kIn; ++i) x[i] = X[static_cast<int64_t>(s) * kIn + i];
  forward_one(sp, x, h1, h2, y);
  Y[s] = y;
}

// Training, per sample: activations H1, H2 and back-propagated deltas of
// L = (1/B) sum_s (y_s - t_s)^2 (dy = dL/dy, D2 = dL/d(pre-tanh 2),
// D1 = dL/d(pre-tanh 1)), and the squared error.
__global__ void __launch_bounds__(kThreads) mlp_deltas_kernel(const double* __restrict__ p,
                                                              const double* __restrict__ X,
                                                              const double* __restrict__ T, int B,
                                                              double* __restrict__ H1, double* __restrict__ H2,
                                                              double* __restrict__ D1, double* __restrict__ D2,
                                                              double* __restrict__ DY, double* __restrict__ SE) {
  __shared__ double sp[kParams];
  for (int t = threadIdx.x; t < kParams; t += kThreads) sp[t] = p[t];
  __syncthreads();
  const int s = blockIdx.x * kThreads + threadIdx.x;
  if (s >= B) return;
  double x[kIn], h1[kH], h2[kH], y;
  for (int i = 0; i < kIn; ++i) x[i] = X[static_cast<int64_t>(s) * kIn + i];
  forward_one(sp, x, h1, h2, y);
  const double e = y - T[s];
  const double dy = 2.0 * e / B;
  double d2[kH];
  for (int i = 0; i < kH; ++i) d2[i] = dy * sp[kOffW3 + i] * (1.0 - h2[i] * h2[i]);
  for (int i = 0; i < kH; ++i) {
    double a = 0.0;
    for (int j = 0; j < kH; ++j) a = fma(d2[j], sp[kOffW2 + j * kH + i], a);
    D1[static_cast<int64_t>(s) * kH + i] = a * (1.0 - h1[i] * h1[i]);
  }
  for (int i = 0; i < kH; ++i) {
    H1[static_cast<int64_t>(s) * kH + i] = h1[i];
    H2[static_cast<int64_t>(s) * kH + i] = h2[i];
    D2[static_cast<int64_t>(s) * kH + i] = d2[i];
  }
  DY[s] = dy;
  SE[s] = e * e;
}

// Training, per parameter q (and the squared-error sum at q = kParams) and
// sample chunk: the chunk's sum of dL/dp_q, samples in order.
__global__ void __launch_bounds__(kThreads) mlp_wgrad_kernel(const double* __restrict__ X,
                                                             const double* __restrict__ H1,
                                                             const double* __restrict__ H2,
                                                             const double* __restrict__ D1,
                                                             const double* __restrict__ D2,
                                                             const double* __restrict__ DY,
                                                             const double* __restrict__ SE, int B, int chunk,
                                                             double* __restrict__ part) {
  const int q = blockIdx.x * kThreads + threadIdx.x;
  if (q > kParams) return;
  const int s0 = blockIdx.y * chunk, s1 = min(B, s0 + chunk);
  double sum = 0.0;
  if (q < kOffB1) {
    const int j = (q - kOffW1) / kIn, i = (q - kOffW1) % kIn;
    for (int s = s0; s < s1; ++s) sum = fma(D1[static_cast<int64_t>(s) * kH + j], X[static_cast<int64_t>(s) * kIn + i], sum);
  } else if (q < kOffW2) {
    const int j = q - kOffB1;
    for (int s = s0; s < s1; ++s) sum += D1[static_cast<int64_t>(s) * kH + j];
  } else if (q < kOffB2) {
    const int j = (q - kOffW2) / kH, i = (q - kOffW2) % kH;
    for (int s = s0; s < s1; ++s) sum = fma(D2[static_cast<int64_t>(s) * kH + j], H1[static_cast<int64_t>(s) * kH + i], sum);
  } else if (q < kOffW3) {
    const int j = q - kOffB2;
    for (int s = s0; s < s1; ++s) sum += D2[static_cast<int64_t>(s) * kH + j];
  } else if (q < kOffB3) {
    const int i = q - kOffW3;
    for (int s = s0; s < s1; ++s) sum = fma(DY[s], H2[static_cast<int64_t>(s) * kH + i], sum);
  } else if (q == kOffB3) {
    for (int s = s0; s < s1; ++s) sum += DY[s];
  } else {
    for (int s = s0; s < s1; ++s) sum += SE[s];
  }
  part[static_cast<int64_t>(blockIdx.y) * (kParams + 1) + q] = sum;
}

__global__ void mlp_reduce_kernel(const double* __restrict__ part, int nparts, double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > kParams) return;
  double sum = 0.0;
  for (int b = 0; b < nparts; ++b) sum += part[static_cast<int64_t>(b) * (kParams + 1) + q];
  out[q] = sum;
}

__global__ void mlp_adam_kernel(double* __restrict__ p, const double* __restrict__ g, double* __restrict__ m,
                                double* __restrict__ v, double lr, double b1, double b2, double eps, double c1,
                                double c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kParams) return;
  const double gq = g[q];
  const double mq = b1 * m[q] + (1.0 - b1) * gq;
  const double vq = b2 * v[q] + (1.0 - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq / c1) / (sqrt(vq / c2) + eps);
}

}  // namespace

struct symla_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  double* d_p = nullptr;
  double* d_m = nullptr;
  double* d_v = nullptr;
  double* d_g = nullptr;     // kParams + 1 (gradient, sum of squared errors)
  double* d_part = nullptr;  // per-chunk partials
  double* d_x = nullptr;
  double* d_t = nullptr;
  double* d_y = nullptr;
  double* d_work = nullptr;  // H1, H2, D1, D2 (B x kH each), DY, SE (B each)
  int batch_cap = 0;
  long long steps = 0;
};

namespace {

int fail(int code, const std::string& msg) { return symla_gpu::record_error(code, msg); }

#define MLP_CK(expr)                                                                          \
  do {                                                                                        \
    const cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess) return fail(SYMLA_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kChunk = 1024;  // samples per gradient chunk

int ensure_batch(symla_mlp* m, int B) {
  if (B <= m->batch_cap) return SYMLA_OK;
  double* ptrs[] = {m->d_x, m->d_t, m->d_y, m->d_part, m->d_work};
  for (double* p : ptrs)
    if (p) cudaFree(p);
  m->d_x = m->d_t = m->d_y = m->d_part = m->d_work = nullptr;
  m->batch_cap = 0;
  const int nparts = (B + kChunk - 1) / kChunk;
  MLP_CK(cudaMalloc(&m->d_x, static_cast<size_t>(B) * kIn * sizeof(double)));
  MLP_CK(cudaMalloc(&m->d_t, static_cast<size_t>(B) * sizeof(double)));
  MLP_CK(cudaMalloc(&m->d_y, static_cast<size_t>(B) * sizeof(double)));
  MLP_CK(cudaMalloc(&m->d_part, static_cast<size_t>(nparts) * (kParams + 1) * sizeof(double)));
  MLP_CK(cudaMalloc(&m->d_work, static_cast<size_t>(B) * (4 * kH + 2) * sizeof(double)));
  m->batch_cap = B;
  return SYMLA_OK;
}

// gradient of the mean squared error over samples [0, B) of the staged
// arrays (offset off) into d_g, d_g[kParams] = sum of squared errors
int grad_staged(symla_mlp* m, int off, int B) {
  const double* X = m->d_x + static_cast<size_t>(off) * kIn;
  const double* T = m->d_t + off;
  double* H1 = m->d_work;
  double* H2 = H1 + static_cast<size_t>(B) * kH;
  double* D1 = H2 + static_cast<size_t>(B) * kH;
  double* D2 = D1 + static_cast<size_t>(B) * kH;
  double* DY = D2 + static_cast<size_t>(B) * kH;
  double* SE = DY + B;
  mlp_deltas_kernel<<<(B + kThreads - 1) / kThreads, kThreads, 0, m->stream>>>(m->d_p, X, T, B, H1, H2, D1, D2, DY,
                                                                                 SE);
  const int nparts = (B + kChunk - 1) / kChunk;
  mlp_wgrad_kernel<<<dim3((kParams + 1 + kThreads - 1) / kThreads, nparts), kThreads, 0, m->stream>>>(
      X, H1, H2, D1, D2, DY, SE, B, kChunk, m->d_part);
  mlp_reduce_kernel<<<(kParams + 1 + 127) / 128, 128, 0, m->stream>>>(m->d_part, nparts, m->d_g);
  MLP_CK(cudaGetLastError());
  return SYMLA_OK;
}

}  // namespace

extern "C" int symla_mlp_create(int device, const double* params, symla_mlp** out) {
  if (!out) return fail(SYMLA_ERR_INVALID, "symla_mlp_create: out is NULL");
  *out = nullptr;
  if (!params) return fail(SYMLA_ERR_INVALID, "symla_mlp_create: params is NULL");
  symla_mlp* m = new symla_mlp();
  m->device = device;
  auto bail = [&](int rc) {
    symla_mlp_destroy(m);
    return rc;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(fail(SYMLA_ERR_NO_DEVICE, "symla_mlp_create: no such CUDA device"));
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&m->d_p, kParams * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&m->d_m, kParams * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&m->d_v, kParams * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&m->d_g, (kParams + 1) * sizeof(double)) != cudaSuccess)
    return bail(fail(SYMLA_ERR_OOM, "symla_mlp_create: device allocation failed"));
  if (cudaMemcpy(m->d_p, params, kParams * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->d_m, 0, kParams * sizeof(double)) != cudaSuccess ||
      cudaMemset(m->d_v, 0, kParams * sizeof(double)) != cudaSuccess)
    return bail(fail(SYMLA_ERR_CUDA, "symla_mlp_create: parameter upload failed"));
  *out = m;
  return SYMLA_OK;
}

extern "C" void symla_mlp_destroy(symla_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  double* ptrs[] = {m->d_p, m->d_m, m->d_v, m->d_g, m->d_part, m->d_x, m->d_t, m->d_y};
  for (double* p : ptrs)
    if (p) cudaFree(p);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

extern "C" int symla_mlp_get_params(symla_mlp* m, double* params) {
  if (!m || !params) return fail(SYMLA_ERR_INVALID, "symla_mlp_get_params: null argument");
  cudaSetDevice(m->device);
  MLP_CK(cudaMemcpyAsync(params, m->d_p, kParams * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  MLP_CK(cudaStreamSynchronize(m->stream));
  return SYMLA_OK;
}

extern "C" int symla_mlp_predict(symla_mlp* m, const double* X, int B, double* Y) {
  if (!m || B < 0 || (B > 0 && (!X || !Y))) return fail(SYMLA_ERR_INVALID, "symla_mlp_predict: bad arguments");
  if (B == 0) return SYMLA_OK;
  cudaSetDevice(m->device);
  int rc = ensure_batch(m, B);
  if (rc != SYMLA_OK) return rc;
  MLP_CK(cudaMemcpyAsync(m->d_x, X, static_cast<size_t>(B) * kIn * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  mlp_forward_kernel<<<(B + kThreads - 1) / kThreads, kThreads, 0, m->stream>>>(m->d_p, m->d_x, B, m->d_y);
  MLP_CK(cudaGetLastError());
  MLP_CK(cudaMemcpyAsync(Y, m->d_y, static_cast<size_t>(B) * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  MLP_CK(cudaStreamSynchronize(m->stream));
  return SYMLA_OK;
}

extern "C" int symla_mlp_gradient(symla_mlp* m, const double* X, const double* T, int B, double* grad, double* loss) {
  if (!m || B <= 0 || !X || !T || !grad) return fail(SYMLA_ERR_INVALID, "symla_mlp_gradient: bad arguments");
  cudaSetDevice(m->device);
  int rc = ensure_batch(m, B);
  if (rc != SYMLA_OK) return rc;
  MLP_CK(cudaMemcpyAsync(m->d_x, X, static_cast<size_t>(B) * kIn * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  MLP_CK(cudaMemcpyAsync(m->d_t, T, static_cast<size_t>(B) * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  rc = grad_staged(m, 0, B);
  if (rc != SYMLA_OK) return rc;
  std::vector<double> h(kParams + 1);
  MLP_CK(cudaMemcpyAsync(h.data(), m->d_g, (kParams + 1) * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  MLP_CK(cudaStreamSynchronize(m->stream));
  for (int q = 0; q < kParams; ++q) grad[q] = h[q];
  if (loss) *loss = h[kParams] / B;
  return SYMLA_OK;
}

extern "C" int symla_mlp_train(symla_mlp* m, const double* X, const double* T, int B, int epochs, int minibatch,
                               double lr, double* final_loss) {
  if (!m || B <= 0 || epochs < 0 || !X || !T) return fail(SYMLA_ERR_INVALID, "symla_mlp_train: bad arguments");
  const int mb = (minibatch <= 0 || minibatch > B) ? B : minibatch;
  cudaSetDevice(m->device);
  int rc = ensure_batch(m, B);
  if (rc != SYMLA_OK) return rc;
  MLP_CK(cudaMemcpyAsync(m->d_x, X, static_cast<size_t>(B) * kIn * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  MLP_CK(cudaMemcpyAsync(m->d_t, T, static_cast<size_t>(B) * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
  for (int e = 0; e < epochs; ++e) {
    for (int off = 0; off < B; off += mb) {
      rc = grad_staged(m, off, std::min(mb, B - off));
      if (rc != SYMLA_OK) return rc;
      ++m->steps;
      const double c1 = 1.0 - std::pow(b1, static_cast<double>(m->steps));
      const double c2 = 1.0 - std::pow(b2, static_cast<double>(m->steps));
      mlp_adam_kernel<<<(kParams + 127) / 128, 128, 0, m->stream>>>(m->d_p, m->d_g, m->d_m, m->d_v, lr, b1, b2, eps,
                                                                     c1, c2);
    }
  }
  MLP_CK(cudaGetLastError());
  if (final_loss) {
    rc = grad_staged(m, 0, B);
    if (rc != SYMLA_OK) return rc;
    double sse = 0.0;
    MLP_CK(cudaMemcpyAsync(&sse, m->d_g + kParams, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MLP_CK(cudaStreamSynchronize(m->stream));
    *final_loss = sse / B;
  }
  MLP_CK(cudaStreamSynchronize(m->stream));
  return SYMLA_OK;
}
