// Supernodal multi-RHS solve kernels (forward, block-diagonal D^{-1},
// backward) walking the tree level by level, plus the FP64 residual used by
// iterative refinement. sm_100a.
//
// Reference behaviour followed (include/symla/...):
//   solve.hpp:303-362  forward: each front gathers its children's forwarded
//                      deltas (RhsElement), solves with its unit-lower Ltop
//                      (d21 slots of 2x2 blocks masked) and forwards
//                      L_bottom * y for its remaining rows to the parent
//   solve.hpp:434-455  D^{-1} with closed-form 2x2 blocks
//   solve.hpp:364-383  backward: gather ancestor values, subtract
//                      L_bottom^T x, transposed unit-lower solve
//   refine.hpp:116     R = B - A.selfadjointView<Lower>() * X
//
// Sign convention: a front's workspace rows for its own pivots hold
// Bp - (children's deltas) - L y, i.e. y after the solve; its remaining rows
// hold the negated forwarded delta, so the parent adds them.
#include <cmath>

#include "common.cuh"
#include "factor_kernels.h"
#include "reduce.cuh"

namespace symla_gpu {

namespace {
constexpr int kSolveThreads = 256;
constexpr int kBlk = 32;
}  // namespace

__global__ void permute_in_kernel(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ B, int ldb,
                                  double* __restrict__ Bp) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(t % n), c = static_cast<int>(t / n);
  Bp[t] = B[perm[i] + static_cast<long long>(c) * ldb];
}

__global__ void permute_out_kernel(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ X,
                                   double* __restrict__ Xout, int ldx) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(t % n), c = static_cast<int>(t / n);
  Xout[perm[i] + static_cast<long long>(c) * ldx] = X[t];
}

__global__ void __launch_bounds__(kSolveThreads) forward_kernel(const FrontDesc* __restrict__ fronts,
                                                                const ChildLink* __restrict__ links,
                                                                const FrontState* __restrict__ st,
                                                                const int* __restrict__ list, int nrhs,
                                                                const double* __restrict__ Bp, double* __restrict__ Z,
                                                                int n) {
  const int s = list[blockIdx.x];
  const FrontDesc f = fronts[s];
  const int m = f.m;
  const int np = st[s].npiv;
  double* W = f.W;
  const int wld = f.wld;
  const int64_t ld = f.ld;
  for (int t = threadIdx.x; t < m * nrhs; t += blockDim.x) {
    const int i = t % m, c = t / m;
    W[i + static_cast<int64_t>(c) * wld] = (i < np) ? Bp[f.fidx[i] + static_cast<int64_t>(c) * n] : 0.0;
  }
  __syncthreads();
  for (int ch = f.ch_begin; ch < f.ch_end; ++ch) {
    const ChildLink L = links[ch];
    const FrontDesc cf = fronts[L.child];
    const int cnp = st[L.child].npiv;
    const int cb = cf.m - cnp;
    for (int t = threadIdx.x; t < cb * nrhs; t += blockDim.x) {
      const int a = t % cb, c = t / cb;
      // relmap gives the parent's pre-pivot position; lpos maps it through
      // the parent's pivoting swaps
      W[f.lpos[L.relmap[a]] + static_cast<int64_t>(c) * wld] += cf.W[cnp + a + static_cast<int64_t>(c) * cf.wld];
    }
    __syncthreads();
  }
  // blocked forward substitution over the pivot columns; rows below each
  // block (own rows and forwarded rows alike) are updated as we go
  for (int j0 = 0; j0 < np; j0 += kBlk) {
    const int j1 = min(j0 + kBlk, np);
    for (int c = threadIdx.x; c < nrhs; c += blockDim.x) {
      double* w = W + static_cast<int64_t>(c) * wld;
      for (int j = j0; j < j1; ++j) {
        const double yj = w[j];
        const double* Lj = f.F + j * ld;
        const int skip = (f.pk[j] == 1) ? j + 1 : -1;
        for (int i = j + 1; i < j1; ++i)
          if (i != skip) w[i] -= Lj[i] * yj;
      }
    }
    __syncthreads();
    const int rows = m - j1;
    for (int t = threadIdx.x; t < rows * nrhs; t += blockDim.x) {
      const int i = j1 + t % rows, c = t / rows;
      double* w = W + static_cast<int64_t>(c) * wld;
      double acc = 0.0;
      for (int j = j0; j < j1; ++j) {
        if (i == j + 1 && f.pk[j] == 1) continue;
        acc += f.F[j * ld + i] * w[j];
      }
      w[i] -= acc;
    }
    __syncthreads();
  }
  // D^{-1}
  for (int t = threadIdx.x; t < np * nrhs; t += blockDim.x) {
    const int q = t % np, c = t / np;
    const double* w = W + static_cast<int64_t>(c) * wld;
    const int8_t kind = f.pk[q];
    if (kind == 0) {
      Z[f.fidx[q] + static_cast<int64_t>(c) * n] = w[q] / f.Dd[q];
    } else if (kind == 1) {
      const double d11 = f.Dd[q], d21 = f.Do[q], d22 = f.Dd[q + 1];
      const double det = d11 * d22 - d21 * d21;
      const double y0 = w[q], y1 = w[q + 1];
      Z[f.fidx[q] + static_cast<int64_t>(c) * n] = (d22 * y0 - d21 * y1) / det;
      Z[f.fidx[q + 1] + static_cast<int64_t>(c) * n] = (-d21 * y0 + d11 * y1) / det;
    }
  }
}

__global__ void __launch_bounds__(kSolveThreads) backward_kernel(const FrontDesc* __restrict__ fronts,
                                                                 const FrontState* __restrict__ st,
                                                                 const int* __restrict__ list, int nrhs,
                                                                 const double* __restrict__ Z, double* __restrict__ X,
                                                                 int n) {
  const int s = list[blockIdx.x];
  const FrontDesc f = fronts[s];
  const int m = f.m;
  const int np = st[s].npiv;
  if (np == 0) return;
  double* W = f.W;
  const int wld = f.wld;
  const int64_t ld = f.ld;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // x_own = z_own - L_bottom^T x_ext   (warp per pivot column)
  for (int q = warp; q < np; q += nwarps) {
    const double* Lq = f.F + q * ld;
    for (int c = 0; c < nrhs; ++c) {
      double acc = 0.0;
      for (int t = np + lane; t < m; t += 32) acc += Lq[t] * X[f.fidx[t] + static_cast<int64_t>(c) * n];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) W[q + static_cast<int64_t>(c) * wld] = Z[f.fidx[q] + static_cast<int64_t>(c) * n] - acc;
    }
  }
  __syncthreads();
  // blocked backward substitution with Ltop^T
  for (int j1 = np; j1 > 0; j1 -= kBlk) {
    const int j0 = max(0, j1 - kBlk);
    // contributions of rows i >= j1 to x[j], j in [j0, j1)
    if (j1 < np) {
      for (int j = j0 + warp; j < j1; j += nwarps) {
        const double* Lj = f.F + j * ld;
        for (int c = 0; c < nrhs; ++c) {
          const double* w = W + static_cast<int64_t>(c) * wld;
          double acc = 0.0;
          for (int i = j1 + lane; i < np; i += 32) {
            if (i == j + 1 && f.pk[j] == 1) continue;
            acc += Lj[i] * w[i];
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
          if (lane == 0) W[j + static_cast<int64_t>(c) * wld] -= acc;
        }
      }
      __syncthreads();
    }
    for (int c = threadIdx.x; c < nrhs; c += blockDim.x) {
      double* w = W + static_cast<int64_t>(c) * wld;
      for (int j = j1 - 1; j >= j0; --j) {
        const double* Lj = f.F + j * ld;
        const int skip = (f.pk[j] == 1) ? j + 1 : -1;
        double acc = 0.0;
        for (int i = j + 1; i < j1; ++i)
          if (i != skip) acc += Lj[i] * w[i];
        w[j] -= acc;
      }
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < np * nrhs; t += blockDim.x) {
    const int q = t % np, c = t / np;
    X[f.fidx[q] + static_cast<int64_t>(c) * n] = W[q + static_cast<int64_t>(c) * wld];
  }
}

__global__ void residual_kernel(int n, int nrhs, const int* __restrict__ rowptr, const int* __restrict__ colind,
                                const int* __restrict__ vidx, const double* __restrict__ vals,
                                const double* __restrict__ X, int ldx, const double* __restrict__ B, int ldb,
                                double* __restrict__ R) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(t % n), c = static_cast<int>(t / n);
  const double* x = X + static_cast<long long>(c) * ldx;
  double acc = 0.0;
  for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) acc += vals[vidx[e]] * x[colind[e]];
  R[i + static_cast<long long>(c) * n] = B[i + static_cast<long long>(c) * ldb] - acc;
}

__global__ void absmax_kernel(const double* __restrict__ v, long long len, double* out) {
  double m = 0.0;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < len;
       t += static_cast<long long>(gridDim.x) * blockDim.x)
    m = fmax(m, fabs(v[t]));
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

__global__ void rowsum_max_kernel(int n, const int* __restrict__ srowptr, const int* __restrict__ svidx,
                                  const double* __restrict__ vals, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < n)
    for (int e = srowptr[i]; e < srowptr[i + 1]; ++e) s += fabs(vals[svidx[e]]);
  s = warp_max(s);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, s);
}

__global__ void axpy_kernel(long long len, const double* __restrict__ dx, double* __restrict__ x) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t < len) x[t] += dx[t];
}

__global__ void copy2d_kernel(int rows, int cols, const double* __restrict__ src, int lds, double* __restrict__ dst,
                              int ldd) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(rows) * cols) return;
  const int i = static_cast<int>(t % rows), c = static_cast<int>(t / rows);
  dst[i + static_cast<long long>(c) * ldd] = src[i + static_cast<long long>(c) * lds];
}

namespace {
inline unsigned grid_for(long long work, int threads) {
  long long g = (work + threads - 1) / threads;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}
}  // namespace

void launch_permute_in(int n, int nrhs, const int* perm, const double* B, int ldb, double* Bp, cudaStream_t stream) {
  permute_in_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, perm, B, ldb, Bp);
}
void launch_permute_out(int n, int nrhs, const int* perm, const double* X, double* Xout, int ldx, cudaStream_t stream) {
  permute_out_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, perm, X, Xout, ldx);
}
void launch_forward(const FrontDesc* fronts, const ChildLink* links, const FrontState* st, const int* list, int count,
                    int nrhs, const double* Bp, double* Z, int n, cudaStream_t stream) {
  if (count <= 0) return;
  forward_kernel<<<count, kSolveThreads, 0, stream>>>(fronts, links, st, list, nrhs, Bp, Z, n);
}
void launch_backward(const FrontDesc* fronts, const FrontState* st, const int* list, int count, int nrhs,
                     const double* Z, double* X, int n, cudaStream_t stream) {
  if (count <= 0) return;
  backward_kernel<<<count, kSolveThreads, 0, stream>>>(fronts, st, list, nrhs, Z, X, n);
}
void launch_residual(int n, int nrhs, const int* rowptr, const int* colind, const int* vidx, const double* vals,
                     const double* X, int ldx, const double* B, int ldb, double* R, cudaStream_t stream) {
  residual_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, rowptr, colind, vidx,
                                                                                       vals, X, ldx, B, ldb, R);
}
void launch_absmax(const double* v, long long len, double* out, cudaStream_t stream) {
  if (len <= 0) return;
  long long g = (len + 255) / 256;
  if (g > 1184) g = 1184;
  absmax_kernel<<<static_cast<unsigned>(g), 256, 0, stream>>>(v, len, out);
}
void launch_rowsum_max(int n, const int* srowptr, const int* svidx, const double* vals, double* out,
                       cudaStream_t stream) {
  if (n <= 0) return;
  rowsum_max_kernel<<<grid_for(n, 256), 256, 0, stream>>>(n, srowptr, svidx, vals, out);
}
void launch_axpy(long long len, const double* dx, double* x, cudaStream_t stream) {
  if (len <= 0) return;
  axpy_kernel<<<grid_for(len, 256), 256, 0, stream>>>(len, dx, x);
}
void launch_copy2d(int rows, int cols, const double* src, int lds, double* dst, int ldd, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return;
  copy2d_kernel<<<grid_for(static_cast<long long>(rows) * cols, 256), 256, 0, stream>>>(rows, cols, src, lds, dst, ldd);
}

}  // namespace symla_gpu
