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
// Work decomposition: every front is cut into 64-row blocks (forward) or
// 64-column blocks of its pivot range (backward). One cooperative launch per
// tree level runs all blocks of all fronts of that level; a block that needs
// the solution of an earlier block of the same front waits for that block's
// flag (release/acquire), so the triangular solve of a large front is
// pipelined across many SMs instead of running in one CTA. Each CTA walks its
// blocks in increasing task order and a block only waits on blocks with a
// smaller task index, and the launch is cooperative (all CTAs resident), so
// the waits always end; every wait is still bounded and reports a timeout
// through the error word instead of spinning forever.
//
// Sign convention: a front's workspace rows for its own pivots hold y after
// the forward pass; its remaining rows hold the negated forwarded delta
// (sum of the children's minus L_bottom * y), so the parent adds them.
#include <cmath>

#include <algorithm>

#include "common.cuh"
#include "factor_kernels.h"
#include "reduce.cuh"

namespace symla_gpu {

namespace {
constexpr int kRB = 64;        // rows (forward) / columns (backward) per block
constexpr int kST = 256;       // threads per CTA
constexpr int kRhsChunk = 16;  // right-hand sides per pass

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Wait until flags[idx] >= epoch; false once wait_ns of the global timer or
// wait_ns / 64 unsuccessful probes (each sleeps 64 ns) have passed (the
// timeout is recorded in the error word), or another CTA raised an error.
__device__ bool wait_flag(const int* flags, int idx, int epoch, int* err, unsigned long long wait_ns) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    if (ld_acquire(flags + idx) < epoch) {
      const unsigned long long t0 = global_ns();
      const unsigned long long max_probes = wait_ns / 64;
      for (unsigned long long it = 1; ld_acquire(flags + idx) < epoch; ++it) {
        if (ld_acquire(err) != 0) {
          ok = 0;
          break;
        }
        if (it > max_probes || global_ns() - t0 > wait_ns) {
          atomicCAS(err, 0, kSolveErrTimeout);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  const bool ok = s_ok != 0;
  __syncthreads();
  return ok;
}

__device__ __forceinline__ void publish(int* flags, int idx, int epoch) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release(flags + idx, epoch);
  }
}
}  // namespace

__global__ void permute_in_kernel(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ B, int ldb,
                                  double* __restrict__ Bp, CheckWord* chk) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(t % n), c = static_cast<int>(t / n);
  const int p = perm[i];
  Bp[t] = check(in_range(p, 0, n), chk, kChkPermute, i) ? B[p + static_cast<long long>(c) * ldb] : 0.0;
}

__global__ void permute_out_kernel(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ X,
                                   double* __restrict__ Xout, int ldx, CheckWord* chk) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  const int i = static_cast<int>(t % n), c = static_cast<int>(t / n);
  const int p = perm[i];
  if (check(in_range(p, 0, n), chk, kChkPermute, i)) Xout[p + static_cast<long long>(c) * ldx] = X[t];
}

// Checked build: a row index or a child workspace row out of range raises
// the solve's error word (the other CTAs then stop waiting) and the access
// is skipped. The ordinary build compiles this to true.
__device__ __forceinline__ bool solve_index_ok(bool ok, int* err) {
  if constexpr (kCheckedBuild) {
    if (!ok) atomicCAS(err, 0, kSolveErrBounds);
    return ok;
  }
  return true;
}

// Shared-memory layout of both pipelined kernels (dynamic, doubles):
//   acc[kRB][kRhsChunk + 1]   the task's result block
//   xb [kRB][kRhsChunk + 1]   the right-hand-side block of the current tile
//   Lb [2][kRB][kRB + 1]      double-buffered L tiles (odd stride: rows and
//                             columns are both conflict-free)
// Every L tile a task needs is known from its position alone, so the next
// tile is copied (cp.async) while the current one is used and before the
// flag that guards its right-hand side is awaited.
constexpr int kAccStride = kRhsChunk + 1;
constexpr int kTileStride = kRB + 1;
constexpr size_t kSolveSmem = (2 * kRB * kAccStride + 2 * kRB * kTileStride) * sizeof(double);

__device__ __forceinline__ void scp_async8(double* smem_dst, const double* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void scp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void scp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Tile (rows [i0, i0 + ni), columns [j0, j0 + nj)) of a front into T,
// T[ii * kTileStride + jj]; entries outside the ranges are zero.
__device__ __forceinline__ void stage_tile(double* T, const double* F, int64_t ld, int i0, int ni, int j0, int nj) {
  for (int t = threadIdx.x; t < kRB * kRB; t += kST) {
    const int ii = t % kRB, jj = t / kRB;
    double* d = T + ii * kTileStride + jj;
    if (ii < ni && jj < nj)
      scp_async8(d, F + static_cast<int64_t>(j0 + jj) * ld + i0 + ii);
    else
      *d = 0.0;
  }
  scp_commit();
}

// ---------------------------------------------------------------------------
// Forward: one row block (front s, block rb). Returns false when a wait
// ended in an error (the CTA then leaves the launch).
__device__ bool forward_block(const FrontDesc* __restrict__ fronts, const ChildLink* __restrict__ links,
                              const FrontState* __restrict__ st, int s, int rb, const int* __restrict__ flag_base,
                              int* flags, int epoch, int* err, unsigned long long wait_ns, int nc, int c0,
                              const double* __restrict__ Bp, int n, double* acc, double* xb, double* Lb0) {
  const int row = threadIdx.x % kRB, cg = threadIdx.x / kRB;  // product layout: a row, 4 right-hand sides
  const FrontDesc f = fronts[s];
  const int m = f.m, np = st[s].npiv;
  const int r0 = rb * kRB, r1 = min(r0 + kRB, m), nr = r1 - r0;
  const int64_t ld = f.ld;
  double* W = f.W;
  const int wld = f.wld;
  const int nbp = (np + kRB - 1) / kRB;
  const int jend = min(rb, nbp);
  const bool hasDiag = r0 < np;
  const int ntiles = jend + (hasDiag ? 1 : 0);
  // pivot kinds the steps below need, loaded before any wait: a 2x2 pivot
  // ending at row r0 - 1 (its d21 slot sits in the last earlier tile) and
  // one starting at this thread's row of the diagonal block
  const bool pair_before = r0 > 0 && r0 - 1 < np && f.pk[r0 - 1] == 1;
  const bool own_pair = hasDiag && threadIdx.x + 1 < min(r1, np) - r0 && f.pk[r0 + threadIdx.x] == 1;
  // tile tt: pivot block tt (tt < jend) or the diagonal block
  auto stage = [&](int tt) {
    double* T = Lb0 + (tt & 1) * kRB * kTileStride;
    if (tt < jend) {
      const int j0 = tt * kRB;
      stage_tile(T, f.F, ld, r0, nr, j0, min(j0 + kRB, np) - j0);
    } else {
      stage_tile(T, f.F, ld, r0, nr, r0, min(r1, np) - r0);
    }
  };
  if (ntiles > 0) stage(0);
  // 1. Bp for pivot rows plus the children's forwarded rows, gathered
  //    through each row's pre-pivot position
  for (int t = threadIdx.x; t < nr * nc; t += kST) {
    const int ii = t % nr, c = t / nr;
    const int i = r0 + ii;
    double v = 0.0;
    if (i < np) {
      const int gi = f.fidx[i];
      if (solve_index_ok(in_range(gi, 0, n), err)) v = Bp[gi + static_cast<int64_t>(c0 + c) * n];
    }
    const int pre = f.lperm[i];
    for (int ch = f.ch_begin; ch < f.ch_end; ++ch) {
      const ChildLink L = links[ch];
      const int a = L.invmap[pre];
      if (a < 0) continue;
      const FrontDesc& cf = fronts[L.child];
      const int cnp = st[L.child].npiv;
      if (solve_index_ok(cnp >= 0 && cnp + a < cf.m, err)) v += cf.W[cnp + a + static_cast<int64_t>(c0 + c) * cf.wld];
    }
    acc[ii * kAccStride + c] = v;
  }
  for (int tt = 0; tt < ntiles; ++tt) {
    const bool more = tt + 1 < ntiles;
    if (more) stage(tt + 1);
    double* T = Lb0 + (tt & 1) * kRB * kTileStride;
    if (tt < jend) {
      // 2. contribution of finished pivot block j = tt
      const int j = tt;
      if (!wait_flag(flags, flag_base[s] + j, epoch, err, wait_ns)) {
        scp_wait<0>();
        return false;
      }
      const int j0 = j * kRB, nj = min(j0 + kRB, np) - j0;
      for (int t = threadIdx.x; t < kRB * nc; t += kST) {
        const int jj = t % kRB, c = t / kRB;
        xb[jj * kAccStride + c] = (jj < nj) ? W[j0 + jj + static_cast<int64_t>(c0 + c) * wld] : 0.0;
      }
      if (more)
        scp_wait<1>();
      else
        scp_wait<0>();
      __syncthreads();
      // a 2x2 pivot straddling the block boundary: its d21 slot in L is not
      // an L entry
      if (threadIdx.x == 0 && j == rb - 1 && r0 - 1 >= j0 && pair_before) T[r0 - 1 - j0] = 0.0;
      __syncthreads();
      if (row < nr) {
        double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
        const int cb4 = cg * 4;
#pragma unroll 8
        for (int jj = 0; jj < nj; ++jj) {
          const double l = T[row * kTileStride + jj];
          const double* y = xb + jj * kAccStride + cb4;
          p0 = fma(l, y[0], p0);
          p1 = fma(l, y[1], p1);
          p2 = fma(l, y[2], p2);
          p3 = fma(l, y[3], p3);
        }
        double* a = acc + row * kAccStride + cb4;
        if (cb4 + 0 < nc) a[0] -= p0;
        if (cb4 + 1 < nc) a[1] -= p1;
        if (cb4 + 2 < nc) a[2] -= p2;
        if (cb4 + 3 < nc) a[3] -= p3;
      }
      __syncthreads();
    } else {
      // 3. the block's own pivot columns: unit-lower solve for its pivot
      //    rows and the matching update of its non-pivot rows
      scp_wait<0>();
      __syncthreads();
      const int npv = min(r1, np) - r0;
      if (own_pair) T[(threadIdx.x + 1) * kTileStride + threadIdx.x] = 0.0;  // d21 slot of a 2x2 pivot
      __syncthreads();
      // a warp takes right-hand sides c and c + 8 together: the two
      // substitution chains interleave (each step is a shuffle and an FMA)
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      constexpr int NW = kST / 32;
      for (int c = warp; c < nc; c += 2 * NW) {
        const int cb = c + NW;
        const bool two = cb < nc;
        double y0 = (lane < nr) ? acc[lane * kAccStride + c] : 0.0;
        double y1 = (lane + 32 < nr) ? acc[(lane + 32) * kAccStride + c] : 0.0;
        double z0 = (two && lane < nr) ? acc[lane * kAccStride + cb] : 0.0;
        double z1 = (two && lane + 32 < nr) ? acc[(lane + 32) * kAccStride + cb] : 0.0;
        for (int jj = 0; jj < npv; ++jj) {
          const double yj = __shfl_sync(0xffffffffu, jj < 32 ? y0 : y1, jj & 31);
          const double zj = __shfl_sync(0xffffffffu, jj < 32 ? z0 : z1, jj & 31);
          const double t0 = T[lane * kTileStride + jj], t1 = T[(lane + 32) * kTileStride + jj];
          if (lane > jj) {
            y0 -= t0 * yj;
            z0 -= t0 * zj;
          }
          if (lane + 32 > jj) {
            y1 -= t1 * yj;
            z1 -= t1 * zj;
          }
        }
        if (lane < nr) acc[lane * kAccStride + c] = y0;
        if (lane + 32 < nr) acc[(lane + 32) * kAccStride + c] = y1;
        if (two && lane < nr) acc[lane * kAccStride + cb] = z0;
        if (two && lane + 32 < nr) acc[(lane + 32) * kAccStride + cb] = z1;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nr * nc; t += kST) {
    const int ii = t % nr, c = t / nr;
    W[r0 + ii + static_cast<int64_t>(c0 + c) * wld] = acc[ii * kAccStride + c];
  }
  if (hasDiag) publish(flags, flag_base[s] + rb, epoch);
  __syncthreads();
  return true;
}

// Forward task = int4 {front, row block, 0, 0}, or {front, -1, 0, 0} for the
// whole front (its row blocks in order, in this CTA). Flag of a pivot row
// block at flag_base[front] + row block.
__global__ void __launch_bounds__(kST, 2) forward_pipelined_kernel(
    const FrontDesc* __restrict__ fronts, const ChildLink* __restrict__ links, const FrontState* __restrict__ st,
    const int4* __restrict__ tasks, int ntasks, const int* __restrict__ flag_base, int* flags, int epoch, int* err,
    unsigned long long wait_ns, int nrhs, int c0, const double* __restrict__ Bp, int n) {
  extern __shared__ double ssm[];
  double* acc = ssm;
  double* xb = acc + kRB * kAccStride;
  double* Lb0 = xb + kRB * kAccStride;
  const int nc = min(kRhsChunk, nrhs - c0);
  for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
    if (ld_acquire(err) != 0) return;
    const int4 tk = tasks[task];
    const int s = tk.x;
    if (tk.y >= 0) {
      if (!forward_block(fronts, links, st, s, tk.y, flag_base, flags, epoch, err, wait_ns, nc, c0, Bp, n, acc, xb, Lb0)) return;
    } else {
      const int nb = (fronts[s].m + kRB - 1) / kRB;
      for (int rb = 0; rb < nb; ++rb)
        if (!forward_block(fronts, links, st, s, rb, flag_base, flags, epoch, err, wait_ns, nc, c0, Bp, n, acc, xb, Lb0))
          return;
    }
  }
}

// ---------------------------------------------------------------------------
// Backward: pivot column block cb of front s. The tiles are the ancestor
// rows [np, m) in 64-row chunks, then the later pivot blocks, then the
// diagonal block. A main part (part 0) does ancestor chunks [a0, a1), the
// later blocks, adds its helper parts' partial sums (slots hslot0 ..
// hslot0 + nh - 1, in slot order) and finishes the block; a helper part
// only sums its ancestor chunks into its scratch slot and raises its flag.
__device__ bool backward_block(const FrontDesc* __restrict__ fronts, const FrontState* __restrict__ st, int s, int cb,
                               bool helper, int a0, int a1, int hslot0, int nh, const int* __restrict__ flag_base,
                               int* flags, int* hflags, double* hscratch, int epoch, int* err,
                               unsigned long long wait_ns, int nc, int c0, double* __restrict__ X, int n, double* acc,
                               double* xb, double* Lb0) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NW = kST / 32;
  const int col = threadIdx.x % kRB, cg = threadIdx.x / kRB;
  const FrontDesc f = fronts[s];
  const int m = f.m, np = st[s].npiv;
  const int q0 = cb * kRB, q1 = min(q0 + kRB, np), nq = q1 - q0;
  const int64_t ld = f.ld;
  const double* W = f.W;
  const int wld = f.wld;
  const int nbp = (np + kRB - 1) / kRB;
  const int nanc = a1 - a0;
  const int nlater = helper ? 0 : nbp - 1 - cb;
  const int ntiles = nanc + nlater + (helper ? 0 : 1);
  // loaded before any wait: the 2x2 pivot kinds the steps below need and
  // the rows the block's solution is written to
  static_assert(kST % kRB == 0, "a thread keeps one tile row in the gathers");
  __shared__ int s_row[kRB];
  const bool pair_at_end = nq > 0 && f.pk[q1 - 1] == 1;
  const bool own_pair = threadIdx.x + 1 < nq && f.pk[q0 + threadIdx.x] == 1;
  if (!helper && threadIdx.x < nq) s_row[threadIdx.x] = f.fidx[q0 + threadIdx.x];
  auto tile_rows = [&](int tt, int& i0, int& i1) {
    if (tt < nanc) {
      i0 = np + (a0 + tt) * kRB;
      i1 = min(i0 + kRB, m);
    } else if (tt < nanc + nlater) {
      const int j = nbp - 1 - (tt - nanc);
      i0 = j * kRB;
      i1 = min(i0 + kRB, np);
    } else {
      i0 = q0;
      i1 = q1;
    }
  };
  auto stage = [&](int tt) {
    int i0, i1;
    tile_rows(tt, i0, i1);
    stage_tile(Lb0 + (tt & 1) * kRB * kTileStride, f.F, ld, i0, i1 - i0, q0, nq);
  };
  if (ntiles > 0) stage(0);
  if (helper) {
    for (int t = threadIdx.x; t < kRB * nc; t += kST) acc[(t % kRB) * kAccStride + t / kRB] = 0.0;
  } else {
    // 1. z = D^{-1} y for the block's pivots (a 2x2 partner may sit in the
    //    neighbouring block; y is complete in W after the forward pass)
    for (int t = threadIdx.x; t < nq * nc; t += kST) {
      const int qq = t % nq, c = t / nq;
      const int q = q0 + qq;
      const double* w = W + static_cast<int64_t>(c0 + c) * wld;
      const int8_t kind = f.pk[q];
      double z;
      if (kind == 0) {
        z = w[q] / f.Dd[q];
      } else if (kind == 1) {
        const double d11 = f.Dd[q], d21 = f.Do[q], d22 = f.Dd[q + 1];
        const double det = d11 * d22 - d21 * d21;
        z = (d22 * w[q] - d21 * w[q + 1]) / det;
      } else {
        const double d11 = f.Dd[q - 1], d21 = f.Do[q - 1], d22 = f.Dd[q];
        const double det = d11 * d22 - d21 * d21;
        z = (-d21 * w[q - 1] + d11 * w[q]) / det;
      }
      acc[qq * kAccStride + c] = z;
    }
  }
  for (int tt = 0; tt < ntiles; ++tt) {
    const bool more = tt + 1 < ntiles;
    if (more) stage(tt + 1);
    double* T = Lb0 + (tt & 1) * kRB * kTileStride;
    int i0, i1;
    tile_rows(tt, i0, i1);
    if (tt < nanc + nlater) {
      // 2. minus L(rows of the tile, block)^T x(rows of the tile): the
      //    ancestor rows are final from earlier levels; later pivot blocks of
      //    this front are waited for
      const int ni = i1 - i0;
      // this thread's tile row (the same for every t below), before the wait
      const int my_ii = threadIdx.x % kRB;
      const int my_gi = my_ii < ni ? f.fidx[i0 + my_ii] : 0;
      if (tt >= nanc) {
        const int j = nbp - 1 - (tt - nanc);
        if (!wait_flag(flags, flag_base[s] + j, epoch, err, wait_ns)) {
          scp_wait<0>();
          return false;
        }
      }
      for (int t = threadIdx.x; t < kRB * nc; t += kST) {
        const int ii = t % kRB, c = t / kRB;
        double xv = 0.0;
        if (ii < ni) {
          const int gi = my_gi;
          if (solve_index_ok(in_range(gi, 0, n), err)) xv = X[gi + static_cast<int64_t>(c0 + c) * n];
        }
        xb[ii * kAccStride + c] = xv;
      }
      if (more)
        scp_wait<1>();
      else
        scp_wait<0>();
      __syncthreads();
      // a 2x2 pivot straddling the block boundary: d21 is not an L entry
      if (threadIdx.x == 0 && i0 == q1 && pair_at_end) T[nq - 1] = 0.0;
      __syncthreads();
      if (col < nq) {
        double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
        const int cb4 = cg * 4;
#pragma unroll 8
        for (int ii = 0; ii < ni; ++ii) {
          const double l = T[ii * kTileStride + col];
          const double* x = xb + ii * kAccStride + cb4;
          p0 = fma(l, x[0], p0);
          p1 = fma(l, x[1], p1);
          p2 = fma(l, x[2], p2);
          p3 = fma(l, x[3], p3);
        }
        double* a = acc + col * kAccStride + cb4;
        if (cb4 + 0 < nc) a[0] -= p0;
        if (cb4 + 1 < nc) a[1] -= p1;
        if (cb4 + 2 < nc) a[2] -= p2;
        if (cb4 + 3 < nc) a[3] -= p3;
      }
      __syncthreads();
    } else {
      // helper parts' partial sums, in slot order (deterministic)
      for (int h = 0; h < nh; ++h) {
        if (!wait_flag(hflags, hslot0 + h, epoch, err, wait_ns)) {
          scp_wait<0>();
          return false;
        }
        const double* part = hscratch + static_cast<int64_t>(hslot0 + h) * kRB * kRhsChunk;
        for (int t = threadIdx.x; t < nq * nc; t += kST) {
          const int qq = t % nq, c = t / nq;
          acc[qq * kAccStride + c] += part[c * kRB + qq];
        }
        __syncthreads();
      }
      // 3. transposed unit-lower solve on the diagonal block
      scp_wait<0>();
      __syncthreads();
      if (own_pair) T[(threadIdx.x + 1) * kTileStride + threadIdx.x] = 0.0;  // d21 slot of a 2x2 pivot
      __syncthreads();
      // right-hand sides c and c + NW together (interleaved chains)
      for (int c = warp; c < nc; c += 2 * NW) {
        const int cb = c + NW;
        const bool two = cb < nc;
        double x0 = (lane < nq) ? acc[lane * kAccStride + c] : 0.0;
        double x1 = (lane + 32 < nq) ? acc[(lane + 32) * kAccStride + c] : 0.0;
        double u0 = (two && lane < nq) ? acc[lane * kAccStride + cb] : 0.0;
        double u1 = (two && lane + 32 < nq) ? acc[(lane + 32) * kAccStride + cb] : 0.0;
        for (int jj = nq - 1; jj >= 0; --jj) {
          // x[jj] is final once every row below it has been applied; row jj
          // of Ltop then updates the unknowns above it
          const double xj = __shfl_sync(0xffffffffu, jj < 32 ? x0 : x1, jj & 31);
          const double uj = __shfl_sync(0xffffffffu, jj < 32 ? u0 : u1, jj & 31);
          const double t0 = T[jj * kTileStride + lane], t1 = T[jj * kTileStride + lane + 32];
          if (lane < jj) {
            x0 -= t0 * xj;
            u0 -= t0 * uj;
          }
          if (lane + 32 < jj) {
            x1 -= t1 * xj;
            u1 -= t1 * uj;
          }
        }
        if (lane < nq) acc[lane * kAccStride + c] = x0;
        if (lane + 32 < nq) acc[(lane + 32) * kAccStride + c] = x1;
        if (two && lane < nq) acc[lane * kAccStride + cb] = u0;
        if (two && lane + 32 < nq) acc[(lane + 32) * kAccStride + cb] = u1;
      }
      __syncthreads();
    }
  }
  if (helper) {
    // acc holds minus the helper's partial sum; the main part adds it
    double* part = hscratch + static_cast<int64_t>(hslot0) * kRB * kRhsChunk;
    for (int t = threadIdx.x; t < nq * nc; t += kST) {
      const int qq = t % nq, c = t / nq;
      part[c * kRB + qq] = acc[qq * kAccStride + c];
    }
    publish(hflags, hslot0, epoch);
  } else {
    for (int t = threadIdx.x; t < nq * nc; t += kST) {
      const int qq = t % nq, c = t / nq;
      const int gi = s_row[qq];
      if (solve_index_ok(in_range(gi, 0, n), err)) X[gi + static_cast<int64_t>(c0 + c) * n] = acc[qq * kAccStride + c];
    }
    publish(flags, flag_base[s] + cb, epoch);
  }
  __syncthreads();
  return true;
}

// Backward task = int4 {front, column block, part, aux}:
//   {s, -1, 0, 0}            the whole front (blocks last to first, this CTA)
//   {s, cb, 0, P << 20 | h0}  main part of block cb with P parts in all; its
//                             helpers hold scratch slots h0 .. h0 + P - 2
//   {s, cb, p, P << 20 | h}   helper part p (1 <= p < P) in slot h
// The ancestor chunks of a block are split evenly over its P parts. Helpers
// are listed before their main part, and later blocks of a front before
// earlier ones, so every wait is on a task with a smaller index.
__global__ void __launch_bounds__(kST, 2) backward_pipelined_kernel(
    const FrontDesc* __restrict__ fronts, const FrontState* __restrict__ st, const int4* __restrict__ tasks,
    int ntasks, const int* __restrict__ flag_base, int* flags, int* hflags, double* hscratch, int epoch, int* err,
    unsigned long long wait_ns, int nrhs, int c0, double* __restrict__ X, int n) {
  extern __shared__ double ssm[];
  double* acc = ssm;
  double* xb = acc + kRB * kAccStride;
  double* Lb0 = xb + kRB * kAccStride;
  const int nc = min(kRhsChunk, nrhs - c0);
  for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
    if (ld_acquire(err) != 0) return;
    const int4 tk = tasks[task];
    const int s = tk.x;
    const int m = fronts[s].m, np = st[s].npiv;
    const int nanc = (m - np + kRB - 1) / kRB;
    if (tk.y < 0) {
      const int nbp = (np + kRB - 1) / kRB;
      for (int cb = nbp - 1; cb >= 0; --cb)
        if (!backward_block(fronts, st, s, cb, false, 0, nanc, 0, 0, flag_base, flags, hflags, hscratch, epoch, err,
                            wait_ns, nc, c0, X, n, acc, xb, Lb0))
          return;
    } else {
      const int P = tk.w >> 20, slot = tk.w & ((1 << 20) - 1), p = tk.z;
      const int a0 = static_cast<int>(static_cast<long long>(nanc) * p / P);
      const int a1 = static_cast<int>(static_cast<long long>(nanc) * (p + 1) / P);
      if (!backward_block(fronts, st, s, tk.y, p > 0, a0, a1, slot, p > 0 ? 1 : P - 1, flag_base, flags, hflags,
                          hscratch, epoch, err, wait_ns, nc, c0, X, n, acc, xb, Lb0))
        return;
    }
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

// The norms of the refinement propagate a NaN (the bit-pattern maximum of
// non-negative values orders NaN above +Inf), so a non-finite residual or
// solution can never read as converged.
__global__ void absmax_kernel(const double* __restrict__ v, long long len, double* out) {
  double m = 0.0;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < len;
       t += static_cast<long long>(gridDim.x) * blockDim.x)
    m = nan_sticky_absmax(m, v[t]);
  m = warp_max_nonneg(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

__global__ void rowsum_max_kernel(int n, const int* __restrict__ srowptr, const int* __restrict__ svidx,
                                  const double* __restrict__ vals, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < n)
    for (int e = srowptr[i]; e < srowptr[i + 1]; ++e) s += fabs(vals[svidx[e]]);
  s = warp_max_nonneg(fabs(s));
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

// ---------------------------------------------------------------------------
// Column-wise vector kernels of GMRES-IR. The Krylov vectors of all
// right-hand sides advance together: vector i, right-hand side c is
// V + i * vs + c * n (n rows, compact).

// partial[(i * nrhs + c) * G + b] = sum over block b's rows of
// V_i[:, c] . W[:, c], with G = gridDim.x; every block sums its rows in a
// fixed order (the host adds the partials in a fixed order too).
__global__ void multi_dot_kernel(int n, int nrhs, const double* __restrict__ V, long long vs,
                                 const double* __restrict__ W, double* __restrict__ partial) {
  __shared__ double red[8];
  const int c = blockIdx.y, i = blockIdx.z;
  const double* v = V + i * vs + static_cast<long long>(c) * n;
  const double* w = W + static_cast<long long>(c) * n;
  double s = 0.0;
  for (long long r = blockIdx.x * 256LL + threadIdx.x; r < n; r += static_cast<long long>(gridDim.x) * 256)
    s = fma(v[r], w[r], s);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += red[k];
    partial[(static_cast<long long>(i) * nrhs + c) * gridDim.x + blockIdx.x] = t;
  }
}

// W[:, c] -= sum_i coef[i * nrhs + c] * V_i[:, c]
__global__ void multi_axpy_kernel(int n, int nrhs, int nvec, const double* __restrict__ V, long long vs,
                                  const double* __restrict__ coef, double* __restrict__ W) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  const int c = static_cast<int>(t / n);
  double acc = W[t];
  for (int i = 0; i < nvec; ++i) acc -= coef[i * nrhs + c] * V[i * vs + t];
  W[t] = acc;
}

// Y[:, c] = alpha[c] * X[:, c]
__global__ void col_scale_kernel(int n, int nrhs, const double* __restrict__ alpha, const double* __restrict__ X,
                                 double* __restrict__ Y) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (t >= static_cast<long long>(n) * nrhs) return;
  Y[t] = alpha[t / n] * X[t];
}

namespace {
inline unsigned grid_for(long long work, int threads) {
  long long g = (work + threads - 1) / threads;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}
}  // namespace

int solve_block_rows() { return kRB; }
int solve_rhs_chunk() { return kRhsChunk; }

cudaError_t solve_max_resident(int device, int* fwd_ctas, int* bwd_ctas) {
  int sms = 0, a = 0, b = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(forward_pipelined_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kSolveSmem));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(backward_pipelined_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kSolveSmem));
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, forward_pipelined_kernel, kST, kSolveSmem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, backward_pipelined_kernel, kST, kSolveSmem);
  if (e != cudaSuccess) return e;
  *fwd_ctas = a * sms;
  *bwd_ctas = b * sms;
  return cudaSuccess;
}

cudaError_t launch_forward_pipelined(const FrontDesc* fronts, const ChildLink* links, const FrontState* st,
                                     const int4* tasks, int ntasks, int grid, const int* flag_base, int* flags,
                                     int epoch, int* err, unsigned long long wait_ns, int nrhs, int c0,
                                     const double* Bp, int n, cudaStream_t stream) {
  if (ntasks <= 0) return cudaSuccess;
  void* args[] = {(void*)&fronts, (void*)&links, (void*)&st,  (void*)&tasks, (void*)&ntasks,
                  (void*)&flag_base, (void*)&flags, (void*)&epoch, (void*)&err, (void*)&wait_ns,
                  (void*)&nrhs, (void*)&c0,     (void*)&Bp,    (void*)&n};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(forward_pipelined_kernel), dim3(grid), dim3(kST),
                                     args, kSolveSmem, stream);
}

cudaError_t launch_backward_pipelined(const FrontDesc* fronts, const FrontState* st, const int4* tasks, int ntasks,
                                      int grid, const int* flag_base, int* flags, int* hflags, double* hscratch,
                                      int epoch, int* err, unsigned long long wait_ns, int nrhs, int c0, double* X,
                                      int n, cudaStream_t stream) {
  if (ntasks <= 0) return cudaSuccess;
  void* args[] = {(void*)&fronts, (void*)&st,    (void*)&tasks, (void*)&ntasks, (void*)&flag_base,
                  (void*)&flags,  (void*)&hflags, (void*)&hscratch, (void*)&epoch, (void*)&err,
                  (void*)&wait_ns, (void*)&nrhs,   (void*)&c0,    (void*)&X,     (void*)&n};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(backward_pipelined_kernel), dim3(grid), dim3(kST),
                                     args, kSolveSmem, stream);
}

void launch_permute_in(int n, int nrhs, const int* perm, const double* B, int ldb, double* Bp, cudaStream_t stream,
                       CheckWord* chk) {
  permute_in_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, perm, B, ldb, Bp,
                                                                                         chk);
}
void launch_permute_out(int n, int nrhs, const int* perm, const double* X, double* Xout, int ldx, cudaStream_t stream,
                        CheckWord* chk) {
  permute_out_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, perm, X, Xout, ldx,
                                                                                          chk);
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
int multi_dot_blocks(int n) { return static_cast<int>(std::min<long long>((n + 255) / 256, 296)); }
void launch_multi_dot(int n, int nrhs, int nvec, const double* V, long long vs, const double* W, double* partial,
                      cudaStream_t stream) {
  if (n <= 0 || nrhs <= 0 || nvec <= 0) return;
  multi_dot_kernel<<<dim3(multi_dot_blocks(n), nrhs, nvec), 256, 0, stream>>>(n, nrhs, V, vs, W, partial);
}
void launch_multi_axpy(int n, int nrhs, int nvec, const double* V, long long vs, const double* coef, double* W,
                       cudaStream_t stream) {
  if (n <= 0 || nrhs <= 0 || nvec <= 0) return;
  multi_axpy_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, nvec, V, vs, coef,
                                                                                        W);
}
void launch_col_scale(int n, int nrhs, const double* alpha, const double* X, double* Y, cudaStream_t stream) {
  if (n <= 0 || nrhs <= 0) return;
  col_scale_kernel<<<grid_for(static_cast<long long>(n) * nrhs, 256), 256, 0, stream>>>(n, nrhs, alpha, X, Y);
}

void launch_copy2d(int rows, int cols, const double* src, int lds, double* dst, int ldd, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return;
  copy2d_kernel<<<grid_for(static_cast<long long>(rows) * cols, 256), 256, 0, stream>>>(rows, cols, src, lds, dst, ldd);
}

}  // namespace symla_gpu
