// Benchmark tooling, not part of the library: the FP64 tensor-path peak of
// this GPU, measured with a register-only loop of independent mma.sync
// m16n8k8 .f64 (DMMA) instructions on every SM, timed with CUDA events. The
// measured copy bandwidth and bf16 GEMM peak that the benchmark's roofline
// uses for HBM- and tensor-bound kernels have no FP64 counterpart, and the
// FP64 Schur update (update_mma_kernel) runs on this pipe, so its roofline
// denominator is taken with the same kind of microbenchmark. Built into its
// own library (libsymla_bench.so), which only bench.py loads.
#include <cuda_runtime.h>

#include <algorithm>

namespace {

constexpr int kPeakWarps = 16;     // warps per CTA
constexpr int kPeakChains = 8;     // independent accumulators per warp
constexpr int kPeakIters = 4096;

__global__ void __launch_bounds__(32 * kPeakWarps) dmma_peak_kernel(double* out) {
  double a[4], b[2], c[kPeakChains][4];
  for (int r = 0; r < 4; ++r) a[r] = 1e-3 * (threadIdx.x + r);
  for (int r = 0; r < 2; ++r) b[r] = 1e-3 * (threadIdx.x - r);
  for (int i = 0; i < kPeakChains; ++i)
    for (int e = 0; e < 4; ++e) c[i][e] = 0.0;
  for (int it = 0; it < kPeakIters; ++it) {
#pragma unroll
    for (int i = 0; i < kPeakChains; ++i)
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
          : "+d"(c[i][0]), "+d"(c[i][1]), "+d"(c[i][2]), "+d"(c[i][3])
          : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
  }
  double s = 0.0;
  for (int i = 0; i < kPeakChains; ++i)
    for (int e = 0; e < 4; ++e) s += c[i][e];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the loop live
}

}  // namespace

// Returns 0 and the peak in TFLOP/s, or the failing cudaError_t.
extern "C" int symla_bench_fp64_tensor_peak(int device, double* tflops) {
  if (!tflops) return static_cast<int>(cudaErrorInvalidValue);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return static_cast<int>(e);
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return static_cast<int>(e);
  const int grid = 2 * sms;
  double* d = nullptr;
  e = cudaMalloc(&d, static_cast<size_t>(grid) * 32 * kPeakWarps * sizeof(double));
  if (e != cudaSuccess) return static_cast<int>(e);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = 0.0f;
  double best = 0.0;
  e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
    e = cudaEventRecord(e0);
    dmma_peak_kernel<<<grid, 32 * kPeakWarps>>>(d);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(e1);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && rep > 0 && ms > 0.0f) {
      const double flops = 2.0 * 16 * 8 * 8 * kPeakChains * static_cast<double>(kPeakIters) * grid * kPeakWarps;
      best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return static_cast<int>(e);
  *tflops = best;
  return 0;
}
