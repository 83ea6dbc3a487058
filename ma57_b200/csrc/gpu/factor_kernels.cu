// Numeric factorization kernels: front assembly (extend + extend-add), dense
// partial LDL^T with threshold Bunch-Kaufman or static pivoting, and the
// Schur-complement (trailing) update. sm_100a.
//
// Reference behaviour followed (include/symla/...):
//   multifrontal.hpp:498-535  F = 0; extend (A entries of own columns);
//                             extend-add of each child's generated element
//   dense_kernel.hpp:576-793  pivot search and 1x1 / swap / 2x2 / delay
//                             decisions, restricted to the eligible rows
//   dense_kernel.hpp:919-1059 static pivoting with sign-matched perturbation
//   dense_kernel.hpp:806-821  trailing update with the panel's L D L^T
//
// Fronts keep only their lower triangle (row >= column); the reference keeps
// both triangles and re-averages them after every update
// (dense_kernel.hpp:269-297), which is a no-op for a computation that forms
// each symmetric entry once.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>

#include "common.cuh"
#include "factor_kernels.h"
#include "reduce.cuh"

namespace symla_gpu {

namespace {

constexpr double kAlpha = 0.64038820320220756;  // (1 + sqrt(17)) / 8

__device__ __forceinline__ bool level_aborted(const FactorGlobals* g, int level, int dynamic) {
  return level_skipped(g, level, dynamic);
}

// Child contribution to parent entry (i, j) (i >= j in the parent's local
// order), summed over children in their fixed order.
__device__ __forceinline__ double gather_children(const FrontDesc* fronts, const ChildLink* links,
                                                  const FrontState* st, int ch_begin, int ch_end, int i, int j,
                                                  CheckWord* chk) {
  double v = 0.0;
  for (int c = ch_begin; c < ch_end; ++c) {
    const ChildLink L = links[c];
    const int b = L.invmap[j];
    if (b < 0) continue;
    const int a = L.invmap[i];
    if (a < 0) continue;
    const FrontDesc& cf = fronts[L.child];
    const int np = st[L.child].npiv;
    const int r = a > b ? a : b, cc = a > b ? b : a;
    if (!check(np >= 0 && np + r < cf.m, chk, kChkGather, L.child)) continue;
    v += cf.F[static_cast<int64_t>(np + cc) * cf.ld + np + r];
  }
  return v;
}

// A stored entry e of the front's own columns: (local column, local row,
// value index), or false (checked build) when it lies outside the front.
__device__ __forceinline__ bool a_entry(const KernelOpts& o, const FrontDesc& f, int e, int& j, int& i, int& idx) {
  j = o.a_j[e];
  const int pos = o.a_pos[e];
  idx = o.a_idx[e];
  i = pos < f.ncols ? pos : pos + f.nextra;
  return check(a_entry_ok(j, pos, idx, f.ncols, f.nextra, f.m, o.nnz), o.chk, kChkAEntry, e);
}

}  // namespace

// ---------------------------------------------------------------------------
// Assembly of large fronts in global memory: one CTA per (front, 32-column
// block, row range); levels with few large fronts split the rows into
// chunks so that they still fill the GPU. Every parent entry is written exactly once (gather
// form), so no separate zero fill and no atomics; then the A entries of the
// block's own columns and rows are added. The children's map pointers, contribution-block
// origins and their maps of the block's 32 columns are staged in shared
// memory once; each thread then takes rows, reads a row's position in each
// child once and issues the (independent) loads of 16 of the 32 columns,
// summing over the children in their fixed order.
namespace {
constexpr int kAsmMaxChildren = 16;
}

__global__ void __launch_bounds__(256, 4) assemble_kernel(const FrontDesc* __restrict__ fronts,
                                                       const ChildLink* __restrict__ links,
                                                       FrontState* st, const int* __restrict__ tasks,
                                                       const int* __restrict__ a_colptr, KernelOpts o,
                                                       const FactorGlobals* __restrict__ g, int level, int dynamic) {
  if (level_aborted(g, level, dynamic)) return;
  __shared__ const int* s_inv[kAsmMaxChildren];
  __shared__ const double* s_cb[kAsmMaxChildren];
  __shared__ int64_t s_ld[kAsmMaxChildren];
  __shared__ int s_b[kAsmMaxChildren][32];
  __shared__ int s_lim[kAsmMaxChildren];  // checked build: contribution-block rows of each child
  const int4 task = reinterpret_cast<const int4*>(tasks)[blockIdx.x];
  const int s = task.x, j0 = task.y, i0 = task.z;  // i0 >= j0
  const FrontDesc f = fronts[s];
  const int j1 = min(j0 + 32, f.m), nj = j1 - j0;
  const int iend = task.w < 0 ? f.m : min(task.w, f.m);
  const int nch = f.ch_end - f.ch_begin;
  if (i0 == j0 && threadIdx.x < nj) f.lperm[j0 + threadIdx.x] = j0 + threadIdx.x;
  if (nch <= kAsmMaxChildren) {
    if (threadIdx.x < nch) {
      const ChildLink L = links[f.ch_begin + threadIdx.x];
      const FrontDesc& cf = fronts[L.child];
      const int np = st[L.child].npiv;
      s_inv[threadIdx.x] = L.invmap;
      s_cb[threadIdx.x] = cf.F + static_cast<int64_t>(np) * cf.ld + np;  // contribution block origin
      s_ld[threadIdx.x] = cf.ld;
      if constexpr (kCheckedBuild)
        s_lim[threadIdx.x] = check(np >= 0 && np <= cf.m, o.chk, kChkPivots, L.child) ? cf.m - np : 0;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nch * 32; t += blockDim.x) {
      const int c = t / 32, jj = t % 32;
      s_b[c][jj] = (jj < nj) ? s_inv[c][j0 + jj] : -1;
    }
    __syncthreads();
    // warp w takes columns j0 + 16 (w & 1) .. + 16 of rows 32 (w >> 1) + lane
    // + 128 t: half a row's loads per thread keeps the registers low enough
    // for four CTAs per SM (the gather is load-latency-bound)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h0 = 16 * (warp & 1);
    for (int i = i0 + 32 * (warp >> 1) + lane; i < iend; i += 128) {
      double acc[16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) acc[jj] = 0.0;
      for (int c = 0; c < nch; ++c) {
        const int a = s_inv[c][i];
        if (a < 0) continue;
        const double* cb = s_cb[c];
        const int64_t cld = s_ld[c];
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const int b = s_b[c][h0 + jj];
          if (b >= 0 && j0 + h0 + jj <= i) {
            const int r = a > b ? a : b, cc = a > b ? b : a;
            if (check(r < s_lim[c], o.chk, kChkGather, s)) acc[jj] += cb[static_cast<int64_t>(cc) * cld + r];
          }
        }
      }
#pragma unroll
      for (int jj = 0; jj < 16; ++jj)
        if (h0 + jj < nj && j0 + h0 + jj <= i) f.F[static_cast<int64_t>(j0 + h0 + jj) * f.ld + i] = acc[jj];
    }
  } else {
    for (int j = j0; j < j1; ++j) {
      double* col = f.F + static_cast<int64_t>(j) * f.ld;
      for (int i = max(j, i0) + threadIdx.x; i < iend; i += blockDim.x)
        col[i] = gather_children(fronts, links, st, f.ch_begin, f.ch_end, i, j, o.chk);
    }
  }
  __syncthreads();
  if (j0 < f.ncols) {
    const int jend = min(j1, f.ncols);
    const int e0 = a_colptr[f.a_begin + j0], e1 = a_colptr[f.a_begin + jend];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      int j, i, idx;
      if (a_entry(o, f, e, j, i, idx) && i >= i0 && i < iend) f.F[static_cast<int64_t>(j) * f.ld + i] += o.values[idx];
    }
  }
  // max |entry| of the assembled front (dense_kernel.hpp:413), folded here
  // so the panel kernel does not rescan the front: a thread takes a row and
  // reads its (up to) 32 entries of the task's columns with independent
  // loads (consecutive rows across a warp), then the next row
  __syncthreads();
  double tmax = 0.0;
  const double* blk = f.F + static_cast<int64_t>(j0) * f.ld;
  for (int i = i0 + threadIdx.x; i < iend; i += blockDim.x) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
#pragma unroll
    for (int jj = 0; jj < 32; jj += 4) {
      const double* p = blk + static_cast<int64_t>(jj) * f.ld + i;
      if (jj + 0 < nj && j0 + jj + 0 <= i) t0 = fmax(t0, fabs(p[0]));
      if (jj + 1 < nj && j0 + jj + 1 <= i) t1 = fmax(t1, fabs(p[f.ld]));
      if (jj + 2 < nj && j0 + jj + 2 <= i) t2 = fmax(t2, fabs(p[2 * static_cast<int64_t>(f.ld)]));
      if (jj + 3 < nj && j0 + jj + 3 <= i) t3 = fmax(t3, fabs(p[3 * static_cast<int64_t>(f.ld)]));
    }
    tmax = fmax(tmax, fmax(fmax(t0, t1), fmax(t2, t3)));
  }
  tmax = warp_max(tmax);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&st[s].orig_max, tmax);
}

// ---------------------------------------------------------------------------
// Small fronts: one CTA per front, the whole front in shared memory
// (assembly, factorization and write-back in one launch).
namespace {

// Warp mode of the small-front kernel: fronts of at most kWarpFrontMax rows,
// kWarpFronts per CTA, each in a fixed slice of kWarpFrontDoubles of the
// dynamic shared memory (the m x (m | 1) front plus its two index arrays).
constexpr int kWarpFrontMax = 32;
constexpr int kWarpFronts = 8;
constexpr int kWarpFrontDoubles = kWarpFrontMax * (kWarpFrontMax | 1) + kWarpFrontMax;

template <int NT>
struct SmallFront {
  double* S;
  int lds;
  int m;
  __device__ double& at(int i, int j) { return S[j * lds + i]; }
  // symmetric read from lower storage
  __device__ double sym(int i, int j) { return i >= j ? S[j * lds + i] : S[i * lds + j]; }
};

// Calls fn(i, j) once for every entry i >= j of a t x t lower triangle,
// spread over the CTA's NT threads. The triangle is folded into a
// (t + 1) x ceil(t / 2) rectangle: rectangle column c holds triangle column
// c (rows c..t-1) in its rows c..t-1 and triangle column t-1-c in the rest
// (rows 0..c-1 -> triangle rows t-c..t-1, row t -> the diagonal), the middle
// column of an odd t only once. Consecutive threads take consecutive
// rectangle rows (consecutive rows of one column: no shared-memory bank
// conflicts), and each thread's position advances by a precomputed step, so
// there is one integer division per call instead of one per entry, and no
// thread idles on the upper half.
template <int NT, class Fn>
__device__ __forceinline__ void for_lower(int t, int tid, Fn&& fn) {
  const int R = t + 1, C = (t + 1) >> 1;
  int q = tid % R, c = tid / R;  // position c R + q, advancing by NT
  const int dq = NT % R, dc = NT / R;
  while (c < C) {
    if (q >= c && q < t) {
      fn(q, c);
    } else {
      const int c2 = t - 1 - c;
      if (c2 != c) fn(q == t ? c2 : c2 + 1 + q, c2);
    }
    q += dq;
    c += dc;
    if (q >= R) {
      q -= R;
      ++c;
    }
  }
}

// The threads that factor one small front: the whole CTA (NT = 128 or 256)
// or one warp (NT = 32; the CTA then holds kWarpFronts fronts, one per
// warp, and no block-wide barrier is used).
template <int NT>
__device__ __forceinline__ void grp_sync() {
  if constexpr (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}
template <int NT>
__device__ __forceinline__ ArgMax grp_argmax(ArgMax a, double* sv, int* si) {
  if constexpr (NT == 32)
    return warp_argmax(a);
  else
    return block_argmax<NT>(a, sv, si);
}
template <int NT>
__device__ __forceinline__ double grp_max(double v, double* sv) {
  if constexpr (NT == 32)
    return warp_max(v);
  else
    return block_max<NT>(v, sv);
}

// Symmetric swap of positions i < j in lower storage over the whole front.
template <int NT>
__device__ void smem_swap(SmallFront<NT>& F, int* fi, int* lp, int i, int j, int tid) {
  const int m = F.m;
  for (int t = tid; t < m - 1; t += NT) {
    if (t < i) {  // row swap in columns c < i
      const int c = t;
      double a = F.at(i, c);
      F.at(i, c) = F.at(j, c);
      F.at(j, c) = a;
    } else if (t < j - 1) {  // c in (i, j): (c, i) <-> (j, c)
      const int c = t + 1;
      double a = F.at(c, i);
      F.at(c, i) = F.at(j, c);
      F.at(j, c) = a;
    } else if (t == j - 1) {  // diagonal
      double a = F.at(i, i);
      F.at(i, i) = F.at(j, j);
      F.at(j, j) = a;
    } else {  // rows r > j
      const int r = t + 1;
      double a = F.at(r, i);
      F.at(r, i) = F.at(r, j);
      F.at(r, j) = a;
    }
  }
  if (tid == 0) {
    int a = fi[i];
    fi[i] = fi[j];
    fi[j] = a;
    a = lp[i];
    lp[i] = lp[j];
    lp[j] = a;
  }
  grp_sync<NT>();
}

}  // namespace

template <int NT>
__global__ void __launch_bounds__(NT == 32 ? 32 * kWarpFronts : NT)
    factor_small_kernel(const FrontDesc* __restrict__ fronts, const ChildLink* __restrict__ links, FrontState* st,
                        const int* __restrict__ front_list, int count, const int* __restrict__ a_colptr, KernelOpts o,
                        FactorGlobals* g, int level, int dynamic) {
  if (level_aborted(g, level, dynamic)) return;
  extern __shared__ double smem_all[];
  __shared__ double red_v[NT / 32];
  __shared__ int red_i[NT / 32];
  // warp mode: warp w of the CTA factors list entry kWarpFronts blockIdx + w
  // in its own slice of shared memory
  const int tid = NT == 32 ? static_cast<int>(threadIdx.x & 31) : static_cast<int>(threadIdx.x);
  const int grp = NT == 32 ? static_cast<int>(threadIdx.x >> 5) : 0;
  const int entry = NT == 32 ? static_cast<int>(blockIdx.x) * kWarpFronts + grp : static_cast<int>(blockIdx.x);
  if (entry >= count) return;  // (warp mode only: the whole warp leaves)
  double* smem = smem_all + (NT == 32 ? static_cast<size_t>(grp) * kWarpFrontDoubles : 0);

  const int s = front_list[entry];
  const FrontDesc f = fronts[s];
  const int m = f.m;
  SmallFront<NT> F{smem, m | 1, m};
  int* fi = reinterpret_cast<int*>(smem + static_cast<size_t>(F.lds) * m);
  int* lp = fi + m;  // local pivot permutation

  // ---- assembly (multifrontal.hpp:498-535), children summed in fixed order
  for_lower<NT>(m, tid, [&](int i, int j) {
    F.at(i, j) = gather_children(fronts, links, st, f.ch_begin, f.ch_end, i, j, o.chk);
  });
  for (int t = tid; t < m; t += NT) {
    fi[t] = f.fidx[t];
    lp[t] = t;
  }
  grp_sync<NT>();
  {
    const int e0 = a_colptr[f.a_begin], e1 = a_colptr[f.a_begin + f.ncols];
    for (int e = e0 + tid; e < e1; e += NT) {
      int j, i, idx;
      if (a_entry(o, f, e, j, i, idx)) F.at(i, j) += o.values[idx];
    }
  }
  grp_sync<NT>();

  // ---- orig_max over the whole front (dense_kernel.hpp:413, :934)
  double tmax = 0.0;
  for_lower<NT>(m, tid, [&](int i, int j) { tmax = fmax(tmax, fabs(F.at(i, j))); });
  double orig_max = grp_max<NT>(tmax, red_v);
  const bool isStatic = (o.mode == 1);
  if (isStatic) {
    if (orig_max < o.static_abs_floor) orig_max = 1.0;
  } else {
    if (orig_max < o.zero_tol) orig_max = 1.0;
  }
  double thread_rmax = 0.0;  // cumulative max of values this thread wrote

  const int effEnd = f.nelig;
  int n_pos = 0, n_neg = 0, n_zero = 0, nPert = 0;
  double pert = 0.0;
  double delta = 0.0;
  int k = 0;

  if (isStatic) {
    // dense_kernel.hpp:919-1059, unblocked (panel_size 1 for small fronts)
    delta = o.front_delta ? o.front_delta[s] : (o.static_delta > 0.0 ? o.static_delta : 1.4901161193847656e-08 * orig_max);
    const double floorv = fmax(o.static_abs_floor, o.static_rel_floor * orig_max);
    // expected sign of the next pivot, loaded one pivot ahead (static
    // pivoting never reorders fi)
    int sign_next = (o.sign_final && effEnd > 0) ? o.sign_final[fi[0]] : 0;
    for (k = 0; k < effEnd; ++k) {
      const double akk = F.at(k, k);
      const int sign = sign_next;
      if (o.sign_final && k + 1 < effEnd) sign_next = o.sign_final[fi[k + 1]];
      bool need;
      if (sign > 0)
        need = akk < floorv;
      else if (sign < 0)
        need = akk > -floorv;
      else
        need = fabs(akk) < floorv;
      double d = akk;
      if (need) {
        const double sg = (sign != 0) ? static_cast<double>(sign) : (akk >= 0.0 ? 1.0 : -1.0);
        d = akk + sg * delta;
        const double applied = d - akk;
        if (applied != 0.0) {
          pert += fabs(applied);
          ++nPert;
        }
      }
      if (d > 0)
        ++n_pos;
      else if (d < 0)
        ++n_neg;
      else
        ++n_zero;
      grp_sync<NT>();
      if (tid == 0) F.at(k, k) = d;
      thread_rmax = fmax(thread_rmax, fabs(d));
      for (int i = k + 1 + tid; i < m; i += NT) {
        const double a = F.at(i, k);
        thread_rmax = fmax(thread_rmax, fabs(a));
        F.at(i, k) = a / d;
      }
      grp_sync<NT>();
      for_lower<NT>(m - k - 1, tid, [&](int ii, int jj) {
        const int i = k + 1 + ii, j = k + 1 + jj;
        const double v = F.at(i, j) - (F.at(i, k) * d) * F.at(j, k);
        F.at(i, j) = v;
        thread_rmax = fmax(thread_rmax, fabs(v));
      });
      grp_sync<NT>();
    }
    for (int t = tid; t < effEnd; t += NT) {
        f.Dd[t] = F.at(t, t);
        f.Do[t] = 0.0;
        f.pk[t] = 0;
      }
  } else {
    // dense_kernel.hpp:576-793, unblocked
    while (k < effEnd) {
      ArgMax am{0.0, -1};
      for (int i = k + 1 + tid; i < effEnd; i += NT) {
        const double v = fabs(F.at(i, k));
        am = argmax_combine(am, ArgMax{v, i});
      }
      am = grp_argmax<NT>(am, red_v, red_i);
      const double lambda = am.v;
      const int r = am.i;
      const double akk = F.at(k, k);
      int dec;  // 0: 1x1 at k, 1: swap k<->r then 1x1, 2: 2x2 (k, r), 3: stop
      if (lambda <= o.zero_tol) {
        const double isolatedFloor = fmax(o.zero_tol, o.rel_floor * orig_max);
        dec = (fabs(akk) <= isolatedFloor) ? 3 : 0;
      } else if (fabs(akk) >= kAlpha * lambda) {
        dec = 0;
      } else {
        double sm = 0.0;
        for (int i = k + tid; i < effEnd; i += NT)
          if (i != r) sm = fmax(sm, fabs(F.sym(i, r)));
        const double sigma = grp_max<NT>(sm, red_v);
        if (fabs(akk) * sigma >= kAlpha * lambda * lambda)
          dec = 0;
        else if (fabs(F.at(r, r)) >= kAlpha * sigma)
          dec = 1;
        else
          dec = 2;
      }
      if (dec == 3) break;
      grp_sync<NT>();
      if (dec == 1) smem_swap<NT>(F, fi, lp, k, r, tid);
      if (dec == 0 || dec == 1) {
        const double d = F.at(k, k);
        if (d > 0)
          ++n_pos;
        else if (d < 0)
          ++n_neg;
        else
          ++n_zero;
        thread_rmax = fmax(thread_rmax, fabs(d));
        for (int i = k + 1 + tid; i < m; i += NT) {
          const double a = F.at(i, k);
          thread_rmax = fmax(thread_rmax, fabs(a));
          F.at(i, k) = a / d;
        }
        if (tid == 0) {
          f.Dd[k] = d;
          f.Do[k] = 0.0;
          f.pk[k] = 0;
        }
        grp_sync<NT>();
        for_lower<NT>(m - k - 1, tid, [&](int ii, int jj) {
          const int i = k + 1 + ii, j = k + 1 + jj;
          const double v = F.at(i, j) - (F.at(i, k) * d) * F.at(j, k);
          F.at(i, j) = v;
          thread_rmax = fmax(thread_rmax, fabs(v));
        });
        grp_sync<NT>();
        k += 1;
        continue;
      }
      // 2x2 pivot
      if (r != k + 1) smem_swap<NT>(F, fi, lp, k + 1, r, tid);
      const double d11 = F.at(k, k), d21 = F.at(k + 1, k), d22 = F.at(k + 1, k + 1);
      const double det = d11 * d22 - d21 * d21;
      const double rm = fmax(orig_max, grp_max<NT>(thread_rmax, red_v));
      const double rm1 = fmax(1.0, rm);
      if (fabs(det) <= o.zero_tol * rm1 * rm1) break;
      thread_rmax = fmax(thread_rmax, fmax(fabs(d11), fmax(fabs(d21), fabs(d22))));
      if (det < 0) {
        ++n_pos;
        ++n_neg;
      } else {
        const double tr = d11 + d22;
        if (tr > 0)
          n_pos += 2;
        else if (tr < 0)
          n_neg += 2;
        else {
          ++n_pos;
          ++n_neg;
        }
      }
      const double inv11 = d22 / det, inv21 = -d21 / det, inv22 = d11 / det;
      for (int i = k + 2 + tid; i < m; i += NT) {
        const double a0 = F.at(i, k), a1 = F.at(i, k + 1);
        thread_rmax = fmax(thread_rmax, fmax(fabs(a0), fabs(a1)));
        F.at(i, k) = a0 * inv11 + a1 * inv21;
        F.at(i, k + 1) = a0 * inv21 + a1 * inv22;
      }
      if (tid == 0) {
        f.Dd[k] = d11;
        f.Dd[k + 1] = d22;
        f.Do[k] = d21;
        f.Do[k + 1] = 0.0;
        f.pk[k] = 1;
        f.pk[k + 1] = 2;
      }
      grp_sync<NT>();
      for_lower<NT>(m - k - 2, tid, [&](int ii, int jj) {
        const int i = k + 2 + ii, j = k + 2 + jj;
        const double l0i = F.at(i, k), l1i = F.at(i, k + 1);
        const double w0 = l0i * d11 + l1i * d21;
        const double w1 = l0i * d21 + l1i * d22;
        const double v = F.at(i, j) - (w0 * F.at(j, k) + w1 * F.at(j, k + 1));
        F.at(i, j) = v;
        thread_rmax = fmax(thread_rmax, fabs(v));
      });
      grp_sync<NT>();
      k += 2;
    }
  }

  // ---- write back (lower triangle of the whole front, permuted indices)
  grp_sync<NT>();
  for_lower<NT>(m, tid, [&](int i, int j) { f.F[static_cast<int64_t>(j) * f.ld + i] = F.at(i, j); });
  for (int t = tid; t < m; t += NT) {
    f.fidx[t] = fi[t];
    f.lperm[t] = lp[t];
    f.lpos[lp[t]] = t;
  }
  const double rmax = grp_max<NT>(thread_rmax, red_v);
    if (tid == 0) {
    FrontState& S = st[s];
    S.npiv = k;
    S.n_pos = n_pos;
    S.n_neg = n_neg;
    S.n_zero = n_zero;
    S.num_perturbed = nPert;
    S.perturb = pert;
    S.orig_max = orig_max;
    S.running_max = fmax(orig_max, rmax);
    S.delta = delta;
    S.k = k;
    int flags = kFlagDone;
    if (k < effEnd) {
      if (f.parent >= 0) {
        flags |= kFlagDelayed;
        atomicMin(&g->delay_level, f.level);
      } else {
        flags |= kFlagSingularRoot;
      }
    } else if (k < m && f.parent < 0) {
      flags |= kFlagSingularRoot;
    }
    S.flags = flags;
  }
}

// ---------------------------------------------------------------------------
// Large fronts: panel of up to NB pivots by one CTA, lazily bringing the
// candidate columns up to date from the front (which holds the panel-start
// state for every non-pivoted column) and the panel's L and D
// (dense_kernel.hpp:516-559). The trailing update follows in
// trailing_update_kernel.
namespace {

constexpr int kPanelThreads = 512;

// Compute current column `col` over rows [k, m) into vec:
// vec[i] = raw(i, col) - sum_q L(i, ps+q) * (D L(col, ps+:))_q
__device__ void panel_current_column(const FrontDesc& f, int ps, int p, int k, int col, double* vec, double* wbuf) {
  // w = D * L(col, ps:ps+p)^T (block diagonal D, 2x2 aware)
  if (threadIdx.x < p) {
    const int q = threadIdx.x;
    const int pq = ps + q;
    const int8_t kind = f.pk[pq];
    const double lq = f.F[static_cast<int64_t>(pq) * f.ld + col];
    double w;
    if (kind == 0) {
      w = f.Dd[pq] * lq;
    } else if (kind == 1) {
      const double l1 = f.F[static_cast<int64_t>(pq + 1) * f.ld + col];
      w = f.Dd[pq] * lq + f.Do[pq] * l1;
    } else {
      const double l0 = f.F[static_cast<int64_t>(pq - 1) * f.ld + col];
      w = f.Do[pq - 1] * l0 + f.Dd[pq] * lq;
    }
    wbuf[q] = w;
  }
  __syncthreads();
  for (int i = k + threadIdx.x; i < f.m; i += blockDim.x) {
    double raw = (i >= col) ? f.F[static_cast<int64_t>(col) * f.ld + i] : f.F[static_cast<int64_t>(i) * f.ld + col];
    double corr = 0.0;
    for (int q = 0; q < p; ++q) corr += f.F[static_cast<int64_t>(ps + q) * f.ld + i] * wbuf[q];
    vec[i] = raw - corr;
  }
  __syncthreads();
}

// Symmetric swap of positions i < j in lower storage over the whole front
// (global memory).
__device__ void global_swap(const FrontDesc& f, int i, int j) {
  const int m = f.m;
  double* F = f.F;
  const int64_t ld = f.ld;
  for (int t = threadIdx.x; t < m - 1; t += blockDim.x) {
    if (t < i) {
      const int c = t;
      double a = F[c * ld + i];
      F[c * ld + i] = F[c * ld + j];
      F[c * ld + j] = a;
    } else if (t < j - 1) {
      const int c = t + 1;
      double a = F[i * ld + c];
      F[i * ld + c] = F[c * ld + j];
      F[c * ld + j] = a;
    } else if (t == j - 1) {
      double a = F[i * ld + i];
      F[i * ld + i] = F[j * ld + j];
      F[j * ld + j] = a;
    } else {
      const int r = t + 1;
      double a = F[i * ld + r];
      F[i * ld + r] = F[j * ld + r];
      F[j * ld + r] = a;
    }
  }
  if (threadIdx.x == 0) {
    int a = f.fidx[i];
    f.fidx[i] = f.fidx[j];
    f.fidx[j] = a;
    a = f.lperm[i];
    f.lperm[i] = f.lperm[j];
    f.lperm[j] = a;
  }
  __syncthreads();
}

}  // namespace

__global__ void __launch_bounds__(kPanelThreads) panel_kernel(const FrontDesc* __restrict__ fronts, FrontState* st,
                                                              const int* __restrict__ front_list, int nb, KernelOpts o,
                                                              FactorGlobals* g, int level, int dynamic,
                                                              double* cols, int cols_stride) {
  if (level_aborted(g, level, dynamic)) return;
  constexpr int NT = kPanelThreads;
  extern __shared__ double smem[];
  __shared__ double red_v[NT / 32];
  __shared__ int red_i[NT / 32];
  __shared__ double wbuf[72];

  const int s = front_list[blockIdx.x];
  const FrontDesc f = fronts[s];
  FrontState S = st[s];
  if (S.flags & kFlagDone) {
    // no panel in this iteration: the updates that follow must do nothing
    if (threadIdx.x == 0) {
      st[s].panel_start = S.k;
      st[s].far = 0;
    }
    return;
  }
  if (S.ob_end == 0 || S.far) {
    S.ob = S.k;
    S.ob_end = min(S.k + kOuterBlock, f.nelig);
    S.far = 0;
    S.flags &= ~kFlagFlush;
  }
  const int m = f.m;
  const int effEnd = f.nelig;
  // the two working columns: shared memory, or this front's slice of the
  // global buffer for fronts too tall for shared memory
  double* colk = cols ? cols + static_cast<size_t>(blockIdx.x) * 2 * cols_stride : smem;
  double* colr = colk + m;

  // First panel: orig_max of the assembled front (from the assembly kernel).
  if (S.k == 0) {
    double om = S.orig_max;
    if (o.mode == 1) {
      if (om < o.static_abs_floor) om = 1.0;
    } else {
      if (om < o.zero_tol) om = 1.0;
    }
    S.orig_max = om;
    S.running_max = om;
    S.n_pos = S.n_neg = S.n_zero = 0;
    S.num_perturbed = 0;
    S.perturb = 0.0;
    S.delta = o.front_delta ? o.front_delta[s] : (o.static_delta > 0.0 ? o.static_delta : 1.4901161193847656e-08 * om);
  }
  const double orig_max = S.orig_max;
  int k = S.k;
  const int ps = k;
  const int pe = ps + min(nb, S.ob_end - ps);
  double thread_rmax = 0.0;
  bool stopped = false;
  bool flush = false;
  int n_pos = S.n_pos, n_neg = S.n_neg, n_zero = S.n_zero, nPert = S.num_perturbed;
  double pert = S.perturb;

  while (k < pe) {
    const int p = k - ps;
    panel_current_column(f, ps, p, k, k, colk, wbuf);
    if (o.mode == 1) {
      const double akk = colk[k];
      const int sign = o.sign_final ? o.sign_final[f.fidx[k]] : 0;
      const double floorv = fmax(o.static_abs_floor, o.static_rel_floor * orig_max);
      bool need;
      if (sign > 0)
        need = akk < floorv;
      else if (sign < 0)
        need = akk > -floorv;
      else
        need = fabs(akk) < floorv;
      double d = akk;
      if (need) {
        const double sg = (sign != 0) ? static_cast<double>(sign) : (akk >= 0.0 ? 1.0 : -1.0);
        d = akk + sg * S.delta;
        const double applied = d - akk;
        if (applied != 0.0) {
          pert += fabs(applied);
          ++nPert;
        }
      }
      if (d > 0)
        ++n_pos;
      else if (d < 0)
        ++n_neg;
      else
        ++n_zero;
      thread_rmax = fmax(thread_rmax, fabs(d));
      for (int i = k + 1 + threadIdx.x; i < m; i += NT) {
        const double a = colk[i];
        thread_rmax = fmax(thread_rmax, fabs(a));
        f.F[static_cast<int64_t>(k) * f.ld + i] = a / d;
      }
      if (threadIdx.x == 0) {
        f.F[static_cast<int64_t>(k) * f.ld + k] = d;
        f.Dd[k] = d;
        f.Do[k] = 0.0;
        f.pk[k] = 0;
      }
      __syncthreads();
      ++k;
      continue;
    }
    ArgMax am{0.0, -1};
    for (int i = k + 1 + threadIdx.x; i < effEnd; i += NT) am = argmax_combine(am, ArgMax{fabs(colk[i]), i});
    am = block_argmax<NT>(am, red_v, red_i);
    const double lambda = am.v;
    const int r = am.i;
    const double akk = colk[k];
    int dec;
    if (lambda <= o.zero_tol) {
      const double isolatedFloor = fmax(o.zero_tol, o.rel_floor * orig_max);
      dec = (fabs(akk) <= isolatedFloor) ? 3 : 0;
    } else if (fabs(akk) >= kAlpha * lambda) {
      dec = 0;
    } else if (r >= S.ob_end && ps > S.ob) {
      dec = 4;  // partner beyond the outer block: apply the deferred update first
    } else {
      panel_current_column(f, ps, p, k, r, colr, wbuf);
      double sm = 0.0;
      for (int i = k + threadIdx.x; i < effEnd; i += NT)
        if (i != r) sm = fmax(sm, fabs(colr[i]));
      const double sigma = block_max<NT>(sm, red_v);
      if (fabs(akk) * sigma >= kAlpha * lambda * lambda)
        dec = 0;
      else if (fabs(colr[r]) >= kAlpha * sigma)
        dec = 1;
      else
        dec = 2;
    }
    if (dec == 3) {
      stopped = true;
      break;
    }
    if (dec == 4) {
      flush = true;
      break;
    }
    __syncthreads();
    if (dec == 0 || dec == 1) {
      double* col = colk;
      if (dec == 1) {
        global_swap(f, k, r);
        // new column k = old column r with rows k and r exchanged
        if (threadIdx.x == 0) {
          const double a = colr[k];
          colr[k] = colr[r];
          colr[r] = a;
        }
        __syncthreads();
        col = colr;
      }
      const double d = col[k];
      if (d > 0)
        ++n_pos;
      else if (d < 0)
        ++n_neg;
      else
        ++n_zero;
      thread_rmax = fmax(thread_rmax, fabs(d));
      for (int i = k + 1 + threadIdx.x; i < m; i += NT) {
        const double a = col[i];
        thread_rmax = fmax(thread_rmax, fabs(a));
        f.F[static_cast<int64_t>(k) * f.ld + i] = a / d;
      }
      if (threadIdx.x == 0) {
        f.F[static_cast<int64_t>(k) * f.ld + k] = d;
        f.Dd[k] = d;
        f.Do[k] = 0.0;
        f.pk[k] = 0;
      }
      __syncthreads();
      k += 1;
      continue;
    }
    // 2x2: bring r to k+1
    if (r != k + 1) {
      global_swap(f, k + 1, r);
      if (threadIdx.x == 0) {
        double a = colk[k + 1];
        colk[k + 1] = colk[r];
        colk[r] = a;
        a = colr[k + 1];
        colr[k + 1] = colr[r];
        colr[r] = a;
      }
      __syncthreads();
    }
    const double d11 = colk[k], d21 = colk[k + 1], d22 = colr[k + 1];
    const double det = d11 * d22 - d21 * d21;
    const double rm = fmax(S.running_max, block_max<NT>(thread_rmax, red_v));
    const double rm1 = fmax(1.0, rm);
    if (fabs(det) <= o.zero_tol * rm1 * rm1) {
      stopped = true;
      break;
    }
    thread_rmax = fmax(thread_rmax, fmax(fabs(d11), fmax(fabs(d21), fabs(d22))));
    if (det < 0) {
      ++n_pos;
      ++n_neg;
    } else {
      const double tr = d11 + d22;
      if (tr > 0)
        n_pos += 2;
      else if (tr < 0)
        n_neg += 2;
      else {
        ++n_pos;
        ++n_neg;
      }
    }
    const double inv11 = d22 / det, inv21 = -d21 / det, inv22 = d11 / det;
    for (int i = k + 2 + threadIdx.x; i < m; i += NT) {
      const double a0 = colk[i], a1 = colr[i];
      thread_rmax = fmax(thread_rmax, fmax(fabs(a0), fabs(a1)));
      f.F[static_cast<int64_t>(k) * f.ld + i] = a0 * inv11 + a1 * inv21;
      f.F[static_cast<int64_t>(k + 1) * f.ld + i] = a0 * inv21 + a1 * inv22;
    }
    if (threadIdx.x == 0) {
      f.F[static_cast<int64_t>(k) * f.ld + k] = d11;
      f.F[static_cast<int64_t>(k) * f.ld + k + 1] = d21;
      f.F[static_cast<int64_t>(k + 1) * f.ld + k + 1] = d22;
      f.Dd[k] = d11;
      f.Dd[k + 1] = d22;
      f.Do[k] = d21;
      f.Do[k + 1] = 0.0;
      f.pk[k] = 1;
      f.pk[k + 1] = 2;
    }
    __syncthreads();
    k += 2;
  }

  const double rmax = block_max<NT>(thread_rmax, red_v);
  if (stopped || k >= effEnd)
    for (int t = threadIdx.x; t < m; t += NT) f.lpos[f.lperm[t]] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    FrontState& W = st[s];
    W.orig_max = orig_max;
    W.delta = S.delta;
    W.running_max = fmax(S.running_max, rmax);
    W.n_pos = n_pos;
    W.n_neg = n_neg;
    W.n_zero = n_zero;
    W.num_perturbed = nPert;
    W.perturb = pert;
    W.panel_start = ps;
    W.k = k;
    W.npiv = k;
    W.ob = S.ob;
    W.ob_end = S.ob_end;
    W.far = (stopped || k >= effEnd || flush || k >= S.ob_end) ? 1 : 0;
    int flags = flush ? kFlagFlush : 0;
    if (stopped || k >= effEnd) {
      flags |= kFlagDone;
      if (k < effEnd) {
        if (f.parent >= 0) {
          flags |= kFlagDelayed;
          atomicMin(&g->delay_level, f.level);
        } else {
          flags |= kFlagSingularRoot;
        }
      } else if (k < m && f.parent < 0) {
        flags |= kFlagSingularRoot;
      }
    }
    W.flags = flags;
  }
}

// ---------------------------------------------------------------------------
// Schur-complement updates of a large front, FP64:
//   near (after every panel): columns [k1, ob_end) of the outer block,
//        pivots [ps, k1) of the panel;
//   far  (after an outer block, a flush or the last panel): columns
//        [max(ob_end, k1), m), pivots [ob, k1) of the whole block.
// C(i, j) -= sum_q L(i, q) (L D)(j, q) for i >= j, over the tiles of every
// front of the level (one tile space).
namespace {
constexpr int kMaxUpdateFronts = 1024;  // fronts per update launch
}  // namespace

__device__ __forceinline__ bool update_range(const FrontState& S, int m, bool far, int& c0, int& c1, int& q0,
                                             int& q1) {
  if (!far) {
    q0 = S.panel_start;
    q1 = S.k;
    c0 = S.k;
    c1 = min(S.ob_end, m);
  } else {
    if (!S.far) return false;
    q0 = S.ob;
    q1 = S.k;
    c0 = max(S.ob_end, S.k);
    c1 = m;
  }
  return q1 > q0 && c1 > c0;
}

// Tiles of front s's update region: column tiles of width tj over [c0, c1),
// each with tm-row tiles from its diagonal down to m.
__device__ __forceinline__ int update_tiles(int m, int c0, int c1, int tj, int tm) {
  int n = 0;
  for (int j = c0; j < c1; j += tj) n += (m - j + tm - 1) / tm;
  return n;
}

// ---------------------------------------------------------------------------
// The near / far updates on the FP64 tensor path: mma.sync m16n8k8 .f64
// (DMMA; the 5th-gen tcgen05 MMA has no FP64 kind). TM x 64 tiles: TM = 128,
// 8 warps of 32 x 32 (2 x 4 MMA tiles, 4 accumulators each per lane), or
// TM = 64 for small fronts, 8 warps of 32 x 16 (the autotuner picks per
// level); two CTAs per SM, so that one CTA's C load and store overlap the
// other's MMAs.
//
// A chunk of 16 pivots of the A rows (L(i, q)) and of the B rows (L(j, q),
// with the 2 x 2 partner columns either side) is staged pivot-major, as the
// front stores it, by bulk copies (cp.async.bulk, one per pivot column, no
// multicast) that one thread issues and an mbarrier per stage counts, in a
// ring of three stages (two chunks in flight). A column's copy starts at the
// even row at or before the tile's first row (16-byte alignment; fronts have
// an even leading dimension) and the tile is read at that parity offset.
// W(j, q) = -(L D)(j, q) is formed once per chunk in shared memory (double
// buffered, D read from global) and the L fragment accumulates onto the C
// tile held in registers: one block barrier per chunk.
namespace {
constexpr int kTJ = 64;   // column tile width
constexpr int kKM = 16;   // K chunk
constexpr int kBS = 68;   // pivot-major stride of the staged B rows and W
constexpr int kMThreads = 256;  // 8 warps
constexpr int kMStages = 3;  // staging ring depth (two chunks in flight)
// pivot-major stride of the staged A rows (doubles): TM + 4 keeps the
// fragment loads conflict-free and holds the parity offset
template <int TM>
constexpr int kAS = TM + 4;
template <int TM>
constexpr size_t mma_smem() {
  return static_cast<size_t>(kMStages * (kKM * kAS<TM> + (kKM + 2) * kBS) + 2 * kKM * kBS) * sizeof(double);
}

// c (16 x 8) += a (16 x 8) * b (8 x 8); lane (g, t) = (lane >> 2, lane & 3):
// a_r = A(g + 8 (r & 1), t + 4 (r >> 1)), b_r = B(t + 4 r, g),
// c_e = C(g + 8 (e >> 1), 2 t + (e & 1))
__device__ __forceinline__ void dmma16x8x8(double* c, const double* a, const double* b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ uint32_t u_smem(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
// Bounded wait for the mbarrier phase `parity`: at most kDefaultWaitNs / 8
// probes (each a few ns or more, so at least about a second); false when
// they run out.
__device__ __forceinline__ bool u_mbar_wait(uint64_t* bar, uint32_t parity) {
  constexpr uint32_t kMaxProbes = static_cast<uint32_t>(kDefaultWaitNs / 8);
  for (uint32_t it = 0; it < kMaxProbes; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(u_smem(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// One bulk copy (no multicast) of `bytes` (a multiple of 16; both addresses
// 16-byte aligned) into this CTA's shared memory, counted on `bar`.
__device__ __forceinline__ void u_copy(double* dst, const double* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(u_smem(dst)),
      "l"(src), "r"(bytes), "r"(u_smem(bar))
      : "memory");
}

// Row ranges of the tile being staged (thread 0 sets them at the tile's
// start; only warp 0 reads them): A rows [ra, ra + na) and B rows
// [rb, rb + nb), both starting on an even row, with na, nb even.
struct UpdateCopyRows {
  int ra, na, rb, nb;
};

// Issue the copies of chunk kc (kn pivots) into one ring stage: A columns
// kc .. kc + kn, B columns kc - 1 .. kc + kn (those inside [q0, q1)), rows
// as in cr. Warp 0: lane 0 registers the bytes on the stage's mbarrier, then
// every lane issues one or two of the (at most 34) column copies.
template <int TM>
__device__ __forceinline__ void u_issue(const double* F, int64_t ld, int q0, int q1, int kc, int kn,
                                        const UpdateCopyRows& cr, double* As, double* Bs, uint64_t* bar, int lane) {
  const int qa = max(kc - 1, q0), qb = min(kc + kn + 1, q1);
  const uint32_t per_a = static_cast<uint32_t>(cr.na) * sizeof(double);
  const uint32_t per_b = static_cast<uint32_t>(cr.nb) * sizeof(double);
  if (lane == 0) {
    const uint32_t total = per_a * kn + per_b * (qb - qa);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(u_smem(bar)), "r"(total) : "memory");
  }
  __syncwarp();
  for (int t = lane; t < kn + (qb - qa); t += 32) {
    if (t < kn)
      u_copy(As + t * kAS<TM>, F + (kc + t) * ld + cr.ra, per_a, bar);
    else
      u_copy(Bs + (qa + t - kn - kc + 1) * kBS, F + (qa + t - kn) * ld + cr.rb, per_b, bar);
  }
}
}  // namespace

template <int MODE, int TM>
__global__ void __launch_bounds__(kMThreads, 2) update_mma_kernel(const FrontDesc* __restrict__ fronts, FrontState* st,
                                                               const int* __restrict__ front_list, int count,
                                                               FactorGlobals* g, int level, int dynamic,
                                                               const double* __restrict__ tc_guard) {
  if (level_aborted(g, level, dynamic)) return;
  constexpr int AS = kAS<TM>;
  constexpr int WROWS = TM / 32;       // warps along the tile's rows
  constexpr int WCOLS = 8 / WROWS;     // warps along its 64 columns
  constexpr int WN = kTJ / WCOLS;      // columns per warp (32 or 16)
  constexpr int CT = WN / 8;           // 8-column MMA tiles per warp
  extern __shared__ __align__(16) double usm[];
  // stage b of the ring: A rows at As_of(b), B rows at Bs_of(b); W double buffered
  auto As_of = [&](int b) { return usm + b * kKM * AS; };
  auto Bs_of = [&](int b) { return usm + kMStages * kKM * AS + b * (kKM + 2) * kBS; };
  auto Ws_of = [&](int b) { return usm + kMStages * (kKM * AS + (kKM + 2) * kBS) + b * kKM * kBS; };
  __shared__ __align__(8) uint64_t full[kMStages];
  __shared__ UpdateCopyRows copy_rows;
  __shared__ int tile_end[2 * kMaxUpdateFronts];
  if (threadIdx.x == 0) {
    for (int b = 0; b < kMStages; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(u_smem(&full[b])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const int nent = (MODE == 2) ? 2 * count : count;
  auto entry_far = [&](int e) { return MODE == 1 || (MODE == 2 && e >= count); };
  for (int t = threadIdx.x; t < nent; t += kMThreads) {
    const int sf = front_list[t % count];
    const bool far = entry_far(t);
    int c0, c1, q0, q1;
    const FrontState S = st[sf];
    bool use = update_range(S, fronts[sf].m, far, c0, c1, q0, q1);
    if (far && use && tc_guard && tc_block_ok(q1 - q0, tc_guard[2 * t], tc_guard[2 * t + 1], g->amax))
      use = false;  // the tensor-core kernel applied this block
    tile_end[t] = use ? update_tiles(fronts[sf].m, c0, c1, kTJ, TM) : 0;
    if (blockIdx.x == 0 && tile_end[t] > 0) {
      const double nc = c1 - c0, mm = fronts[sf].m;
      const double entries = nc * mm - (static_cast<double>(c0) + c1 - 1) * nc / 2.0;
      atomicAdd(far ? &g->flops_far : &g->flops_near, 2.0 * (q1 - q0) * entries);
    }
  }
  __shared__ int scan_tot[kMThreads / 32];
  block_inclusive_scan<kMThreads, 2 * kMaxUpdateFronts / kMThreads>(tile_end, nent, scan_tot);
  const int total = nent > 0 ? tile_end[nent - 1] : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = warp / WCOLS, wc = warp % WCOLS;   // warp's 32 x WN sub-tile
  const int lg = lane >> 2, lt = lane & 3;          // fragment coordinates
  double tmax = 0.0;
  int cur = -1, s = -1;
  const double* Fp = nullptr;
  int m = 0, c0 = 0, c1 = 0, q0 = 0, q1 = 0, nchunks = 0;
  int64_t ld = 0;
  unsigned u = 0;  // chunks consumed by this CTA so far (ring stage u % 3, phase (u / 3) & 1)
  // the CTA's tiles increase, so the entry fi, its column tile tj and that
  // column tile's first tile (tj_first, counted within the entry) only move
  // forward: each is advanced from where the previous tile left it
  int fi = 0, tj = 0, tj_first = 0;
  // rows of a tile's copies, from the even row at or before its first row,
  // rounded up to whole 16-byte pairs (the extra row of an odd m is the
  // padding row of the front's even leading dimension); warp 0
  auto set_copy_rows = [&](int ti0, int tj0, int tm) {
    if (lane == 0) {
      copy_rows.ra = ti0 & ~1;
      copy_rows.na = ((min(ti0 + TM, tm) + 1) & ~1) - copy_rows.ra;
      copy_rows.rb = tj0 & ~1;
      copy_rows.nb = ((min(tj0 + kTJ, tm) + 1) & ~1) - copy_rows.rb;
    }
    __syncwarp();
  };
  // the CTA's next tile nt: its first (up to two) chunks into stages
  // (u + 1) % 3 and (u + 2) % 3, issued by warp 0 after the barrier of this
  // tile's last chunk u (every warp is past the chunks that used those
  // stages). The walk runs on copies: the tile loop repeats it at nt.
  auto issue_next = [&](int nt) {
    int nfi = fi, ntj = tj, ntjf = tj_first;
    while (nt >= tile_end[nfi]) {
      ++nfi;
      ntj = 0;
      ntjf = 0;
    }
    const int ns = front_list[nfi % count];
    const int nm = fronts[ns].m;
    int nc0, nc1, nq0, nq1;
    update_range(st[ns], nm, entry_far(nfi), nc0, nc1, nq0, nq1);
    const int nrel = nt - (nfi > 0 ? tile_end[nfi - 1] : 0);
    for (;;) {
      const int nr = (nm - (nc0 + ntj * kTJ) + TM - 1) / TM;
      if (nrel < ntjf + nr) break;
      ntjf += nr;
      ++ntj;
    }
    const int nj0 = nc0 + ntj * kTJ, ni0 = nj0 + (nrel - ntjf) * TM;
    set_copy_rows(ni0, nj0, nm);
    const int nn = (nq1 - nq0 + kKM - 1) / kKM;
    for (int cc = 0; cc < 2 && cc < nn; ++cc) {
      const int kc = nq0 + cc * kKM;
      const unsigned b = (u + 1 + cc) % kMStages;
      u_issue<TM>(fronts[ns].F, fronts[ns].ld, nq0, nq1, kc, min(kKM, nq1 - kc), copy_rows, As_of(b), Bs_of(b),
                  &full[b], lane);
    }
  };
  bool ahead = false;  // warp 0 issued this tile's first chunks during the previous tile
  for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
    while (tile >= tile_end[fi]) {
      ++fi;
      tj = 0;
      tj_first = 0;
    }
    if (fi != cur) {
      if (cur >= 0) {
        tmax = warp_max(tmax);
        if (lane == 0) atomic_max_nonneg(&st[s].running_max, tmax);
        tmax = 0.0;
      }
      cur = fi;
      s = front_list[fi % count];
      Fp = fronts[s].F;
      m = fronts[s].m;
      ld = fronts[s].ld;
      update_range(st[s], m, entry_far(fi), c0, c1, q0, q1);
      nchunks = (q1 - q0 + kKM - 1) / kKM;
    }
    const int rel = tile - (fi > 0 ? tile_end[fi - 1] : 0);
    for (;;) {
      const int nr = (m - (c0 + tj * kTJ) + TM - 1) / TM;
      if (rel < tj_first + nr) break;
      tj_first += nr;
      ++tj;
    }
    const int j0 = c0 + tj * kTJ, i0 = j0 + (rel - tj_first) * TM;
    const int sa = i0 & 1, sb = j0 & 1;  // parity offsets of the staged rows
    __syncthreads();  // previous tile done with every stage and with W
    if (warp == 0 && !ahead) {
      set_copy_rows(i0, j0, m);
      for (int c = 0; c < 2 && c < nchunks; ++c) {
        const int kc = q0 + c * kKM;
        const unsigned b = (u + c) % kMStages;
        u_issue<TM>(Fp, ld, q0, q1, kc, min(kKM, q1 - kc), copy_rows, As_of(b), Bs_of(b), &full[b], lane);
      }
    }
    ahead = false;
    // C tile into the accumulators (lane holds rows gi0 + 16 rt + 8 v,
    // columns gj0 + 8 ct + h as acc[rt][ct][2 v + h])
    const int gi0 = i0 + wr * 32 + lg, gj0 = j0 + wc * WN + 2 * lt;
    double acc[2][CT][4];
#pragma unroll
    for (int ct = 0; ct < CT; ++ct)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gj = gj0 + ct * 8 + h;
        const double* colp = Fp + static_cast<int64_t>(gj < c1 ? gj : 0) * ld;
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int v = 0; v < 2; ++v) {
            const int gi = gi0 + rt * 16 + 8 * v;
            acc[rt][ct][2 * v + h] = (gj < c1 && gi < m && gi >= gj) ? colp[gi] : 0.0;
          }
      }
    // D of this thread's pivot of a chunk (pivot q = threadIdx.x / 16 of the
    // chunk; W row q, columns (threadIdx.x % 16) + 16 j): loaded one chunk
    // ahead into registers, so no global load waits between a chunk's
    // staging and its barrier
    const int wq = threadIdx.x >> 4, wr0 = threadIdx.x & 15;
    int dk = 0;
    double dd = 0.0, dn = 0.0, dp = 0.0;
    auto load_d = [&](int kc, int kn) {
      if (wq < kn) {
        const FrontDesc& fd = fronts[s];
        const int pq = kc + wq;
        dk = fd.pk[pq];
        dd = fd.Dd[pq];
        dn = fd.Do[pq];
        dp = pq > 0 ? fd.Do[pq - 1] : 0.0;
      }
    };
    load_d(q0, min(kKM, q1 - q0));
    for (int c = 0; c < nchunks; ++c, ++u) {
      const int kc = q0 + c * kKM, kn = min(kKM, q1 - kc);
      const unsigned b = u % kMStages;
      if (!u_mbar_wait(&full[b], (u / kMStages) & 1)) {
        // a copy did not land within the wait limit: record it (the
        // factorization then fails with a timeout) and wait once more,
        // bounded, for this stage's copies before going on
        atomicCAS(&g->error, 0, kUpdateErrTimeout);
        u_mbar_wait(&full[b], (u / kMStages) & 1);
      }
      double* As = As_of(b);
      const double* Bs = Bs_of(b) + sb;
      double* Ws = Ws_of(c & 1);
      // the MMAs run over 8-pivot steps: A columns past kn are zeroed (the
      // stage's copies did not write them), W rows past kn are zero
      const int kn8 = (kn + 7) & ~7;
      for (int t = threadIdx.x; t < (kn8 - kn) * AS; t += kMThreads) As[kn * AS + t] = 0.0;
      // W(j, q) = -(L D)(j, q)
      if (wq < kn8) {
#pragma unroll
        for (int j = 0; j < kTJ / 16; ++j) {
          const int r = wr0 + 16 * j;
          double w = 0.0;
          if (wq < kn) {
            const double* col = Bs + (wq + 1) * kBS + r;
            w = dd * col[0];
            if (dk == 1) w += dn * col[kBS];
            if (dk == 2) w += dp * col[-kBS];
          }
          Ws[wq * kBS + r] = -w;
        }
      }
      __syncthreads();  // W and the zeroed columns ready; every thread is past chunk c - 1
      if (c + 1 < nchunks) load_d(kc + kKM, min(kKM, q1 - kc - kKM));
      if (warp == 0 && c + 2 < nchunks) {
        const int kc2 = kc + 2 * kKM;
        const unsigned b2 = (u + 2) % kMStages;
        u_issue<TM>(Fp, ld, q0, q1, kc2, min(kKM, q1 - kc2), copy_rows, As_of(b2), Bs_of(b2), &full[b2], lane);
      } else if (warp == 0 && c == nchunks - 1 && tile + static_cast<int>(gridDim.x) < total) {
        issue_next(tile + static_cast<int>(gridDim.x));
        ahead = true;
      }
      const double* Aq = As + sa;
      for (int k0 = 0; k0 < kn8; k0 += 8) {
        double bq[CT][2];
#pragma unroll
        for (int ct = 0; ct < CT; ++ct)
#pragma unroll
          for (int r = 0; r < 2; ++r) bq[ct][r] = Ws[(k0 + lt + 4 * r) * kBS + wc * WN + ct * 8 + lg];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) {
          double a[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) a[r] = Aq[(k0 + lt + 4 * (r >> 1)) * AS + wr * 32 + rt * 16 + lg + 8 * (r & 1)];
#pragma unroll
          for (int ct = 0; ct < CT; ++ct) dmma16x8x8(acc[rt][ct], a, bq[ct]);
        }
      }
    }
#pragma unroll
    for (int ct = 0; ct < CT; ++ct)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gj = gj0 + ct * 8 + h;
        double* colp = const_cast<double*>(Fp) + static_cast<int64_t>(gj < c1 ? gj : 0) * ld;
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int v = 0; v < 2; ++v) {
            const int gi = gi0 + rt * 16 + 8 * v;
            if (gj < c1 && gi < m && gi >= gj) {
              colp[gi] = acc[rt][ct][2 * v + h];
              tmax = fmax(tmax, fabs(acc[rt][ct][2 * v + h]));
            }
          }
      }
  }
  if (cur >= 0) {
    tmax = warp_max(tmax);
    if (lane == 0) atomic_max_nonneg(&st[s].running_max, tmax);
  }
}

// ---------------------------------------------------------------------------
// Host launchers

void launch_assemble(const FrontDesc* fronts, const ChildLink* links, FrontState* st, const int* tasks,
                     int ntasks, const int* a_colptr, const KernelOpts& o, const FactorGlobals* g, int level,
                     int dynamic, cudaStream_t stream) {
  if (ntasks <= 0) return;
  assemble_kernel<<<ntasks, 256, 0, stream>>>(fronts, links, st, tasks, a_colptr, o, g, level, dynamic);
}

size_t small_front_smem(int m) {
  return static_cast<size_t>(m | 1) * m * sizeof(double) + 2 * static_cast<size_t>(m) * sizeof(int) + 16;
}

void launch_factor_small(const FrontDesc* fronts, const ChildLink* links, FrontState* st, const int* list, int count,
                         int max_m, const int* a_colptr, const KernelOpts& o, FactorGlobals* g, int level, int dynamic,
                         cudaStream_t stream, int threads) {
  if (count <= 0) return;
  const size_t sm = small_front_smem(max_m);
  if (max_m <= kWarpFrontMax && (threads == 32 || threads == 0)) {
    // one warp per front, kWarpFronts fronts per CTA
    const int grid = (count + kWarpFronts - 1) / kWarpFronts;
    factor_small_kernel<32><<<grid, 32 * kWarpFronts, kWarpFronts * kWarpFrontDoubles * sizeof(double), stream>>>(
        fronts, links, st, list, count, a_colptr, o, g, level, dynamic);
  } else if (threads == 128 || (threads != 256 && max_m <= 48)) {
    factor_small_kernel<128><<<count, 128, sm, stream>>>(fronts, links, st, list, count, a_colptr, o, g, level,
                                                          dynamic);
  } else {
    factor_small_kernel<256><<<count, 256, sm, stream>>>(fronts, links, st, list, count, a_colptr, o, g, level,
                                                          dynamic);
  }
}

// Dynamic shared memory the single-CTA panel kernel is configured for.
constexpr size_t kPanelSmemMax = 200 * 1024;

bool panel_fits_shared(int max_m) { return 2 * static_cast<size_t>(max_m) * sizeof(double) <= kPanelSmemMax; }

cudaError_t launch_panel(const FrontDesc* fronts, FrontState* st, const int* list, int count, int max_m, int nb,
                         const KernelOpts& o, FactorGlobals* g, int level, int dynamic, cudaStream_t stream,
                         double* cols) {
  if (count <= 0) return cudaSuccess;
  if (!panel_fits_shared(max_m) && !cols) return cudaErrorInvalidValue;
  const size_t sm = cols ? 0 : 2 * static_cast<size_t>(max_m) * sizeof(double);
  panel_kernel<<<count, kPanelThreads, sm, stream>>>(fronts, st, list, nb, o, g, level, dynamic, cols, max_m);
  return cudaGetLastError();
}


__global__ void count_unfinished_kernel(const FrontState* __restrict__ st, const int* __restrict__ list, int count,
                                        int* out) {
  int c = 0;
  for (int t = threadIdx.x; t < count; t += blockDim.x)
    if (!(st[list[t]].flags & kFlagDone)) ++c;
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

void launch_count_unfinished(const FrontState* st, const int* list, int count, int* out, cudaStream_t stream) {
  if (count <= 0) return;
  count_unfinished_kernel<<<1, 256, 0, stream>>>(st, list, count, out);
}

// Graph launches: a level with an unfinished front after its planned
// iterations marks itself, so the later levels of the graph return at once.
__global__ void mark_unfinished_kernel(const FrontState* __restrict__ st, const int* __restrict__ list, int count,
                                       FactorGlobals* g, int level) {
  if (level_skipped(g, level, 0)) return;
  int c = 0;
  for (int t = threadIdx.x; t < count; t += blockDim.x)
    if (!(st[list[t]].flags & kFlagDone)) ++c;
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicMin(&g->unfinished_level, level);
}

void launch_mark_unfinished(const FrontState* st, const int* list, int count, FactorGlobals* g, int level,
                            cudaStream_t stream) {
  if (count <= 0) return;
  mark_unfinished_kernel<<<1, 256, 0, stream>>>(st, list, count, g, level);
}

namespace {
template <int MODE, int TM>
void launch_update_t(const FrontDesc* fronts, FrontState* st, const int* list, int count, int grid_x,
                     FactorGlobals* g, int level, int dynamic, cudaStream_t stream, const double* tc_guard) {
  for (int b = 0; b < count; b += kMaxUpdateFronts) {
    const int cnt = count - b < kMaxUpdateFronts ? count - b : kMaxUpdateFronts;
    update_mma_kernel<MODE, TM><<<grid_x, kMThreads, mma_smem<TM>(), stream>>>(
        fronts, st, list + b, cnt, g, level, dynamic, (MODE == 1 && tc_guard) ? tc_guard + 2 * b : nullptr);
  }
}
}  // namespace

void launch_update(bool far, const FrontDesc* fronts, FrontState* st, const int* list, int count, int grid_x,
                   FactorGlobals* g, int level, int dynamic, cudaStream_t stream, const double* tc_guard,
                   int tile_rows) {
  if (count <= 0 || grid_x <= 0) return;
  grid_x = std::min(2 * grid_x, 2 * 148);  // two tiles per 128 x 128, two CTAs per SM
  if (tile_rows == 64) {
    if (far)
      launch_update_t<1, 64>(fronts, st, list, count, grid_x, g, level, dynamic, stream, tc_guard);
    else
      launch_update_t<0, 64>(fronts, st, list, count, grid_x, g, level, dynamic, stream, nullptr);
  } else {
    if (far)
      launch_update_t<1, 128>(fronts, st, list, count, grid_x, g, level, dynamic, stream, tc_guard);
    else
      launch_update_t<0, 128>(fronts, st, list, count, grid_x, g, level, dynamic, stream, nullptr);
  }
}

void launch_update_both(const FrontDesc* fronts, FrontState* st, const int* list, int count, int grid_x,
                        FactorGlobals* g, int level, int dynamic, cudaStream_t stream, int tile_rows) {
  if (count <= 0 || grid_x <= 0) return;
  grid_x = std::min(2 * grid_x, 2 * 148);  // two tiles per 128 x 128, two CTAs per SM
  if (tile_rows == 64)
    launch_update_t<2, 64>(fronts, st, list, count, grid_x, g, level, dynamic, stream, nullptr);
  else
    launch_update_t<2, 128>(fronts, st, list, count, grid_x, g, level, dynamic, stream, nullptr);
}

// ---------------------------------------------------------------------------
// Table validation of the checked build: one CTA per front of the list (or
// of all fronts). Phase 0 (before the level launches): descriptor shape,
// storage inside one of the front allocations, row indices, child links and
// their maps, the front's A entries. Phase 1 (after the factorization): the
// pivot counts and the (now permuted) row indices. Phase 2 (before a solve):
// the row indices and the solve workspace slice. Reads the tables only.
__global__ void validate_fronts_kernel(const FrontDesc* __restrict__ fronts, const ChildLink* __restrict__ links,
                                       const FrontState* __restrict__ st, const int* __restrict__ list,
                                       int num_fronts, int n, const int* __restrict__ a_colptr, KernelOpts o,
                                       const double* const* __restrict__ ranges, int nranges, const double* wlo,
                                       const double* whi, int wcols, int phase) {
  __shared__ int s_ok;
  const int s = list ? list[blockIdx.x] : static_cast<int>(blockIdx.x);
  CheckWord* chk = o.chk;
  if (threadIdx.x == 0) {
    bool ok = check(in_range(s, 0, num_fronts), chk, kChkFrontShape, s);
    if (ok) {
      const FrontDesc f = fronts[s];
      ok = check(front_shape_ok(f.m, f.ld, f.ncols, f.nelig, f.nextra), chk, kChkFrontShape, s);
      if (ok) {
        bool inside = false;
        for (int r = 0; r < nranges && !inside; ++r) inside = storage_ok(f.F, f.m, f.ld, ranges[2 * r], ranges[2 * r + 1]);
        ok = check(inside, chk, kChkFrontStorage, s);
      }
      if (ok && phase == 0)
        ok = check(in_range(f.a_begin, 0, n + 1) && f.a_begin + f.ncols <= n && f.ch_begin <= f.ch_end, chk,
                   kChkFrontShape, s);
      if (ok && phase == 1) ok = check(in_range(st[s].npiv, 0, f.nelig + 1), chk, kChkPivots, s);
      if (ok && phase == 2)
        ok = check(f.wld >= f.m && storage_ok(f.W, wcols, f.wld, wlo, whi), chk, kChkWorkspace, s);
    }
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  const FrontDesc f = fronts[s];
  for (int i = threadIdx.x; i < f.m; i += blockDim.x) check(in_range(f.fidx[i], 0, n), chk, kChkRowIndex, s);
  if (phase != 0) return;
  for (int c = f.ch_begin; c < f.ch_end; ++c) {
    const ChildLink L = links[c];
    if (!check(in_range(L.child, 0, num_fronts) && L.child != s, chk, kChkChildLink, s)) continue;
    if (!check(L.cb >= 0 && L.cb <= fronts[L.child].m, chk, kChkChildLink, L.child)) continue;
    for (int i = threadIdx.x; i < f.m; i += blockDim.x) check(in_range(L.invmap[i], -1, L.cb), chk, kChkInvMap, s);
    for (int i = threadIdx.x; i < L.cb; i += blockDim.x) check(in_range(L.relmap[i], 0, f.m), chk, kChkRelMap, s);
  }
  const int e0 = a_colptr[f.a_begin], e1 = a_colptr[f.a_begin + f.ncols];
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    int j, i, idx;
    a_entry(o, f, e, j, i, idx);
  }
}

void launch_validate_fronts(const FrontDesc* fronts, const ChildLink* links, const FrontState* st, const int* list,
                            int count, int num_fronts, int n, const int* a_colptr, const KernelOpts& o,
                            const double* const* ranges, int nranges, const double* wlo, const double* whi,
                            int wcols, int phase, cudaStream_t stream) {
  if (count <= 0) return;
  validate_fronts_kernel<<<count, 256, 0, stream>>>(fronts, links, st, list, num_fronts, n, a_colptr, o, ranges,
                                                     nranges, wlo, whi, wcols, phase);
}

cudaError_t configure_factor_kernels() {
  cudaError_t e;
  e = cudaFuncSetAttribute(factor_small_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kWarpFronts * kWarpFrontDoubles * sizeof(double)));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(factor_small_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(factor_small_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kPanelSmemMax));
  if (e != cudaSuccess) return e;
  for (auto fn : {update_mma_kernel<0, 128>, update_mma_kernel<1, 128>, update_mma_kernel<2, 128>}) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(mma_smem<128>()));
    if (e != cudaSuccess) return e;
  }
  for (auto fn : {update_mma_kernel<0, 64>, update_mma_kernel<1, 64>, update_mma_kernel<2, 64>}) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(mma_smem<64>()));
    if (e != cudaSuccess) return e;
  }
  return e;
}

}  // namespace symla_gpu
