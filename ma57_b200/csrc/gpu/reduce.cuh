// Block-level reductions used by the dense kernels.
#pragma once

#include <cuda_runtime.h>

namespace symla_gpu {

// (value, index) argmax with the reference's scan semantics: the larger value
// wins; among equal values the smaller index wins (dense_kernel.hpp:588-596
// scans rows upward with a strict '>').
struct ArgMax {
  double v;
  int i;
};

__device__ __forceinline__ ArgMax argmax_combine(ArgMax a, ArgMax b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i && b.i >= 0)) return b;
  return a;
}

__device__ __forceinline__ ArgMax warp_argmax(ArgMax a) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    ArgMax o;
    o.v = __shfl_xor_sync(0xffffffffu, a.v, off);
    o.i = __shfl_xor_sync(0xffffffffu, a.i, off);
    a = argmax_combine(a, o);
  }
  return a;
}

// Block argmax; every thread returns the result. Scratch: NT/32 entries each.
template <int NT>
__device__ __forceinline__ ArgMax block_argmax(ArgMax a, double* sv, int* si) {
  a = warp_argmax(a);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    sv[wid] = a.v;
    si[wid] = a.i;
  }
  __syncthreads();
  ArgMax r{sv[0], si[0]};
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) r = argmax_combine(r, ArgMax{sv[w], si[w]});
  return r;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* sv) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sv[wid] = v;
  __syncthreads();
  double r = sv[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) r = fmax(r, sv[w]);
  return r;
}

// Warp max of non-negative doubles (NaN, whose pattern is larger, wins):
// the bit patterns order like the values, so two 32-bit reductions on the
// high and then the low word give the exact maximum.
__device__ __forceinline__ double warp_max_nonneg(double v) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
  const unsigned hi = static_cast<unsigned>(b >> 32), lo = static_cast<unsigned>(b);
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
  return __longlong_as_double(static_cast<long long>((static_cast<unsigned long long>(mh) << 32) | ml));
}

// atomicMax for non-negative doubles (IEEE order == integer order there). A
// NaN is kept (its pattern orders above +Inf), so a maximum over values that
// include a NaN reads NaN instead of a finite number.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  if (v < 0.0) return;
  atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// max(m, |x|) that keeps a NaN once one was seen (fmax would drop it).
__device__ __forceinline__ double nan_sticky_absmax(double m, double x) {
  const double a = fabs(x);
  return (a > m || a != a) ? (m != m ? m : a) : m;
}

// In-place inclusive prefix sum of a[0, n) (n <= PER * NT) by the whole CTA
// of NT threads: each thread sums PER consecutive entries, the per-thread
// sums are scanned with warp shuffles and one pass over the warp totals,
// and each thread rewrites its entries. Every thread must call it; it starts
// and ends with a block barrier.
template <int NT, int PER>
__device__ __forceinline__ void block_inclusive_scan(int* a, int n, int* warp_tot) {
  static_assert(NT % 32 == 0 && NT / 32 <= 32, "block size");
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b0 = threadIdx.x * PER;
  int loc = 0;
#pragma unroll
  for (int i = 0; i < PER; ++i)
    if (b0 + i < n) loc += a[b0 + i];
  int x = loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < NT / 32 ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < NT / 32) warp_tot[lane] = w;
  }
  __syncthreads();
  int run = x - loc + (warp > 0 ? warp_tot[warp - 1] : 0);
#pragma unroll
  for (int i = 0; i < PER; ++i)
    if (b0 + i < n) {
      run += a[b0 + i];
      a[b0 + i] = run;
    }
  __syncthreads();
}

}  // namespace symla_gpu
