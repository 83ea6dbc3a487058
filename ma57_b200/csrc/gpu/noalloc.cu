// Relative residual of a candidate solution with no device allocation.
//
// symla_gpu_solve_refine measures ||B - A X||_inf / (||A||_inf ||X||_inf +
// ||B||_inf) with the residual R and four norm accumulators in buffers that
// the context allocates with cudaMalloc when it first sees a given number of
// right-hand sides. Callers whose device memory is owned by another
// allocator (a fixed budget handed out by a host framework) or whose loop
// cannot take the device-wide synchronisation of cudaMalloc / cudaFree need
// the same measure without those calls. This file gives it to them: the
// same residual and reduction kernels run with their scratch in one
// file-scope device array of fixed size, which every GPU that loads the
// library keeps until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../../include/symla_gpu.h"
#include "context.hpp"
#include "factor_kernels.h"

namespace {

// 4 norm accumulators (padded to 32 doubles = 256 B) + R, n x nrhs doubles.
constexpr long long kNormSlots = 32;
constexpr long long kResidualMax = SYMLA_NOALLOC_RESIDUAL_MAX_ENTRIES;
static __device__ __align__(256) double g_residual_scratch[kNormSlots + kResidualMax];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device; the host-side symbol itself is not a device address).
cudaError_t scratch_on(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_residual_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

int fail(int code, const std::string& msg) { return symla_gpu::record_error(code, msg); }

}  // namespace

extern "C" int symla_gpu_relative_residual_noalloc(symla_gpu_ctx* c, const double* X, int ldx, const double* B,
                                                   int ldb, int nrhs, double* rel_residual) {
  using namespace symla_gpu;
  if (!c || !c->factorized)
    return fail(SYMLA_ERR_NOT_FACTORIZED, "symla_gpu_relative_residual_noalloc: factorize() must be called first");
  if (!rel_residual) return fail(SYMLA_ERR_INVALID, "symla_gpu_relative_residual_noalloc: rel_residual is NULL");
  const int n = c->n;
  if (nrhs < 0 || ldx < n || ldb < n)
    return fail(SYMLA_ERR_BAD_SIZE, "symla_gpu_relative_residual_noalloc: ldx and ldb must be at least n");
  const long long len = static_cast<long long>(n) * nrhs;
  if (len > kResidualMax)
    return fail(SYMLA_ERR_BAD_SIZE, "symla_gpu_relative_residual_noalloc: n * nrhs = " + std::to_string(len) +
                                        " exceeds the fixed scratch of " + std::to_string(kResidualMax) +
                                        " entries (SYMLA_NOALLOC_RESIDUAL_MAX_ENTRIES)");
  if (len == 0) {
    *rel_residual = 0.0;
    return SYMLA_OK;
  }
  if (!X || !B) return fail(SYMLA_ERR_INVALID, "symla_gpu_relative_residual_noalloc: X or B is NULL");
  if (c->device < 0 || c->device >= kMaxDevices)
    return fail(SYMLA_ERR_INVALID, "symla_gpu_relative_residual_noalloc: device index out of range");
  cudaError_t e = cudaSetDevice(c->device);
  double* scratch = nullptr;
  if (e == cudaSuccess) e = scratch_on(c->device, &scratch);
  if (e != cudaSuccess)
    return fail(SYMLA_ERR_CUDA, std::string("symla_gpu_relative_residual_noalloc: ") + cudaGetErrorString(e));
  cudaStream_t st = c->stream;
  double* norms = scratch;            // [0] ||A||_inf, [1] max|B|, [2] max|R|, [3] max|X|
  double* R = scratch + kNormSlots;  // n x nrhs, leading dimension n
  // The accumulators keep the previous call's maxima: clear them first.
  e = cudaMemsetAsync(norms, 0, 4 * sizeof(double), st);
  if (e == cudaSuccess) {
    launch_rowsum_max(n, c->d_srowptr, c->d_svidx, c->d_values, norms + 0, st);
    launch_residual(n, nrhs, c->d_rowptr, c->d_colind, c->d_vidx, c->d_values, X, ldx, B, ldb, R, st);
    launch_absmax(R, len, norms + 2, st);
    for (int j = 0; j < nrhs; ++j) {
      launch_absmax(B + static_cast<long long>(j) * ldb, n, norms + 1, st);
      launch_absmax(X + static_cast<long long>(j) * ldx, n, norms + 3, st);
    }
    e = cudaGetLastError();
  }
  double h[4] = {0.0, 0.0, 0.0, 0.0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, norms, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return fail(SYMLA_ERR_CUDA, std::string("symla_gpu_relative_residual_noalloc: ") + cudaGetErrorString(e));
  const double denom = h[0] * h[3] + h[1];
  *rel_residual = denom > 0.0 ? h[2] / denom : h[2];
  return SYMLA_OK;
}
