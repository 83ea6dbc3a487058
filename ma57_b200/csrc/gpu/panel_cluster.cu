// Panel factorization of large fronts by a thread-block cluster.
//
// One cluster of CS CTAs (2, 4, 8 or 16) factors up to NB pivots of one front.
// The rows [ps, m) of the front are split into CS contiguous slices; CTA q
// keeps, in its shared memory, the panel's L values of its rows (one column
// per pivot of the panel) and the current values of the candidate columns.
// Per pivot every CTA brings its rows of column k up to date
// (raw - L_panel * D * L_panel(k, :)^T, dense_kernel.hpp:516-545), reduces
// its part of the eligible-row argmax, and the partial results are exchanged
// through distributed shared memory; every CTA then takes the same
// Bunch-Kaufman decision (dense_kernel.hpp:576-793). Two cluster barriers per
// pivot in the common (1x1 at k) case.
//
// The front in global memory holds the panel-start ("raw") values of every
// non-pivoted column; row/column interchanges are applied to it and to the
// shared-memory copies. The near and far updates of the panel follow in
// update_kernel / the tensor-core far update.
//
// Speculative panel. Most pivots of most fronts are 1x1 pivots at k (the
// Bunch-Kaufman test |a_kk| >= alpha * lambda passes), and the test can be
// checked after the fact: factor the panel without pivoting, then compare
// each pivot with lambda = max over the eligible rows of its column's
// current values, which the unpivoted factorization produces exactly (the
// same left-looking sums as the sequential path). Every CTA factors the
// panel's diagonal block redundantly in shared memory (no exchange needed
// for D and the L rows of the block), then its own rows below the block in
// one pass with no per-pivot synchronisation; the per-pivot partial lambdas
// cross the cluster once. The pivots before the first one that fails are
// accepted (identical values and decisions to the sequential path), and
// the same launch finishes the panel on the sequential path from the first
// failing pivot (measured: cheaper than a new panel + update launch pair).
#include <cooperative_groups.h>

#include <cmath>

#include "common.cuh"
#include "factor_kernels.h"
#include "reduce.cuh"

namespace cg = cooperative_groups;

namespace symla_gpu {

namespace {

constexpr double kAlphaBK = 0.64038820320220756;  // (1 + sqrt(17)) / 8
constexpr int kCT = 256;                           // threads per CTA
constexpr int kNBMax = 34;                         // panel width + 2
constexpr int kSpecMax = 32;                       // pivots per speculative panel (= panel width)
constexpr int kSpecRetry = 2;                      // consecutive failed panel starts before one sequential decision first
constexpr int kStageHalf = (kNBMax / 2) * (kNBMax / 2 + 1);  // >= np * p0 of any restart (np + p0 <= kNBMax)

struct ClusterShared {
  double w[kNBMax];     // D * L(k, :)^T for the current pivot row
  double wr[kNBMax];    // D * L(r, :)^T for the partner row
  double Dd[kNBMax], Do[kNBMax];
  int pk[kNBMax];
  double ex_v[16];      // per-CTA partial maxima (slow path)
  int ex_i[16];         // per-CTA argmax rows (slow path)
  double ex_x[4];       // values broadcast by the owner of a row (slow path)
  // fast path, double-buffered by step parity: partial argmax per CTA, the
  // pivot's diagonal, and row k+1's current value, sign and panel L row
  double fx_v[2][16];
  int fx_i[2][16];
  double fx_kk[2];
  int fx_sign[2];
  double fx_k1[2];
  double fx_row[2][kNBMax];
  double red_v[kCT / 32];
  int red_i[kCT / 32];
  double rowtmp[kNBMax];  // D * L(row, :) staging
  double rowA[kNBMax], rowB[kNBMax];  // row interchange staging
  double vA[2], vB[2];
  // speculative panel
  double db[kSpecMax][kSpecMax + 1];  // diagonal block: raw lower triangle -> L, d on the diagonal
  double wv[kSpecMax][kSpecMax + 1];  // wv[c][t] = d_t * L(c, t), t < c
  double aabs[kSpecMax][kSpecMax + 1];  // |current value| of the diagonal-block column entries
  double dv[kSpecMax], iv[kSpecMax];  // pivots (after static perturbation) and 1 / pivot
  double pv[kSpecMax];                // applied perturbation (static mode)
  double lamd[kSpecMax], rmd[kSpecMax];  // diagonal-block rows: lambda part, running-max part
  double lamw[kCT / 32][kSpecMax], rvw[kCT / 32][kSpecMax];  // per warp, rows below the block
  double lamx[16][kSpecMax];          // per CTA partial lambda (exchange)
  int kstar;                          // accepted speculative pivots
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long pc_global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bulk (TMA, non-tensor, no multicast) global -> own shared memory copy of
// `bytes` (a multiple of 16; both addresses 16-byte aligned), completing on
// the mbarrier's transaction count.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait for the mbarrier phase `parity` (at most kDefaultWaitNs of the
// global timer, and as many probes); false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const unsigned long long t0 = pc_global_ns();
  for (unsigned long long it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it > kDefaultWaitNs / 8 || ((it & 255) == 255 && pc_global_ns() - t0 > kDefaultWaitNs)) return false;
  }
}

// 8-byte asynchronous global -> shared copy (no register round trip, so
// the copies of a staging loop are all in flight at once)
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most the newest group of this thread's copies is in flight
__device__ __forceinline__ void cp_async_wait_but_newest() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

}  // namespace

template <int CS>
__global__ void __launch_bounds__(kCT) cluster_panel_kernel(const FrontDesc* __restrict__ fronts, FrontState* st,
                                                            const int* __restrict__ front_list, int nb, int R,
                                                            KernelOpts o, FactorGlobals* g, int level, int dynamic) {
  if (level_skipped(g, level, dynamic)) return;
  cg::cluster_group cluster = cg::this_cluster();
  const int q = static_cast<int>(cluster.block_rank());
  const int s = front_list[blockIdx.x / CS];
  const FrontDesc f = fronts[s];
  FrontState S = st[s];
  if (S.flags & kFlagDone) {
    if (q == 0 && threadIdx.x == 0) {
      st[s].panel_start = S.k;
      st[s].far = 0;
    }
    return;
  }
  // outer block bookkeeping: a new block starts at the first panel and after
  // every far update (the far kernel of the previous iteration ran)
  if (S.ob_end == 0 || S.far) {
    S.ob = S.k;
    S.ob_end = min(S.k + kOuterBlock, f.nelig);
    S.far = 0;
    S.flags &= ~kFlagFlush;
  }
  extern __shared__ __align__(16) double dsm[];
  __shared__ __align__(8) uint64_t rows_bar;  // bulk staging of the rows below the block
  __shared__ ClusterShared sh;
  const int m = f.m, effEnd = f.nelig;
  const int64_t ld = f.ld;
  double* F = f.F;
  const int ps = S.k;
  const int pe = ps + min(nb, S.ob_end - ps);
  const int span = m - ps;
  const int Rr = (span + CS - 1) / CS;  // rows per CTA (<= R)
  const int base = ps + q * Rr;
  const int rend = min(base + Rr, m);
  // Lr (column-major, Lr[col * R + li]), vk and vr start at the parity of
  // this CTA's first row, so that a row's slot and its column entry in the
  // front (16-byte aligned columns: even leading dimension) share their
  // 16-byte alignment and whole columns can be staged by bulk copies; R is
  // even with a spare slot past the last row.
  auto lr_of = [&](int rank) { return dsm + ((ps + rank * Rr) & 1); };
  double* Lr = lr_of(q);
  double* vk = Lr + static_cast<size_t>(nb + 2) * R;
  double* vr = vk + R;
  double* stage = dsm + 2 + static_cast<size_t>(nb + 4) * R;  // speculation restarts (2 kStageHalf)
  uint32_t rows_phase = 0;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&rows_bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  auto owner = [&](int i) { return (i - ps) / Rr; };
  auto remote = [&](auto* p, int rank) { return cluster.map_shared_rank(p, rank); };

  // ---- orig_max over the whole front at the first panel (cluster-wide)
  if (ps == 0) {
    // max |entry| of the assembled front, accumulated by the assembly kernel
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
  for (int t = threadIdx.x; t < (kCT / 32) * kSpecMax; t += kCT) {
    sh.lamw[t / kSpecMax][t % kSpecMax] = 0.0;
    sh.rvw[t / kSpecMax][t % kSpecMax] = 0.0;
  }
  int n_pos = S.n_pos, n_neg = S.n_neg, n_zero = S.n_zero, nPert = S.num_perturbed;
  double pert = S.perturb;
  double thread_rmax = S.running_max;  // includes orig_max at the first panel
  double rm_known = S.running_max;

  // compute current values of column `col` for this CTA's rows >= k
  auto current_column = [&](int col, int k, int p, const double* w, double* v) {
    for (int i = max(base, k) + threadIdx.x; i < rend; i += kCT) {
      const int li = i - base;
      const double raw = (i >= col) ? F[col * ld + i] : F[i * ld + col];
      double acc = 0.0;
      for (int t = 0; t < p; ++t) acc += Lr[t * R + li] * w[t];
      v[li] = raw - acc;
    }
  };
  // D * L(row, 0:p)^T from the owner's shared copy (block diagonal D)
  auto d_times_row = [&](int row, int p, double* out) {
    const int li = row - base;
    for (int t = threadIdx.x; t < p; t += kCT) {
      const int kind = sh.pk[t];
      const double lt = Lr[t * R + li];
      double v;
      if (kind == 0)
        v = sh.Dd[t] * lt;
      else if (kind == 1)
        v = sh.Dd[t] * lt + sh.Do[t] * Lr[(t + 1) * R + li];
      else
        v = sh.Do[t - 1] * Lr[(t - 1) * R + li] + sh.Dd[t] * lt;
      out[t] = v;
    }
  };
  // symmetric interchange of positions a < b: global front, row indices and
  // the shared copies of both rows / current values
  auto interchange = [&](int a, int b, bool swapVr) {
    // global front: split the m-1 index range over the cluster
    for (int t = q * kCT + threadIdx.x; t < m - 1; t += CS * kCT) {
      if (t < a) {
        const int c = t;
        double x = F[c * ld + a];
        F[c * ld + a] = F[c * ld + b];
        F[c * ld + b] = x;
      } else if (t < b - 1) {
        const int c = t + 1;
        double x = F[a * ld + c];
        F[a * ld + c] = F[c * ld + b];
        F[c * ld + b] = x;
      } else if (t == b - 1) {
        double x = F[a * ld + a];
        F[a * ld + a] = F[b * ld + b];
        F[b * ld + b] = x;
      } else {
        const int r = t + 1;
        double x = F[a * ld + r];
        F[a * ld + r] = F[b * ld + r];
        F[b * ld + r] = x;
      }
    }
    if (q == 0 && threadIdx.x == 0) {
      int x = f.fidx[a];
      f.fidx[a] = f.fidx[b];
      f.fidx[b] = x;
      x = f.lperm[a];
      f.lperm[a] = f.lperm[b];
      f.lperm[b] = x;
    }
    // shared copies: each owner stages the partner row (a CTA owning both
    // rows stages both), then writes after a barrier
    const int oa = owner(a), ob = owner(b);
    auto stage_row = [&](int row, double* dst, double* vdst) {
      const int oo = owner(row);
      const int lo = row - (ps + oo * Rr);
      double* Lo = remote(lr_of(oo), oo);
      const double* vko = Lo + static_cast<size_t>(nb + 2) * R;
      const double* vro = vko + R;
      for (int t = threadIdx.x; t < nb + 2; t += kCT) dst[t] = Lo[static_cast<size_t>(t) * R + lo];
      if (threadIdx.x == 0) {
        vdst[0] = vko[lo];
        vdst[1] = vro[lo];
      }
    };
    if (q == oa) stage_row(b, sh.rowB, sh.vB);
    if (q == ob) stage_row(a, sh.rowA, sh.vA);
    __threadfence();
    cluster.sync();
    auto write_row = [&](int row, const double* src, const double* vsrc) {
      const int li = row - base;
      for (int t = threadIdx.x; t < nb + 2; t += kCT) Lr[static_cast<size_t>(t) * R + li] = src[t];
      if (threadIdx.x == 0) {
        vk[li] = vsrc[0];
        if (swapVr) vr[li] = vsrc[1];
      }
    };
    if (q == oa) write_row(a, sh.rowB, sh.vB);
    if (q == ob) write_row(b, sh.rowA, sh.vA);
    __threadfence();
    cluster.sync();
  };

  int k = ps;
  bool stopped = false;
  bool flush = false;
  int step = 0;

  // prefetched raw values of column k for this thread's rows
  constexpr int kPF = 4;
  double pf[kPF];
  int pf_col = -1;
  auto prefetch = [&](int col, int kfrom) {
    int j = 0;
    for (int i = max(base, kfrom) + threadIdx.x; i < rend && j < kPF; i += kCT, ++j)
      pf[j] = (i >= col) ? F[col * ld + i] : F[i * ld + col];
    pf_col = col;
  };
  auto current_column_pf = [&](int col, int kk, int p, const double* w, double* v) {
    int j = 0;
    for (int i = max(base, kk) + threadIdx.x; i < rend; i += kCT, ++j) {
      const int li = i - base;
      double raw;
      if (pf_col == col && j < kPF)
        raw = pf[j];
      else
        raw = (i >= col) ? F[col * ld + i] : F[i * ld + col];
      double acc = 0.0;
      for (int t = 0; t < p; ++t) acc += Lr[t * R + li] * w[t];
      v[li] = raw - acc;
    }
  };
  // new w for row k+1 after a 1x1 pivot d at panel position p, from the
  // broadcast L row of k+1 and its current value vk1
  auto local_w_next = [&](int p, double d, const double* lrow, double vk1) {
    for (int t = threadIdx.x; t <= p; t += kCT) {
      double v;
      if (t == p) {
        v = d * (vk1 * (1.0 / d));
      } else {
        const int kind = sh.pk[t];
        if (kind == 0)
          v = sh.Dd[t] * lrow[t];
        else if (kind == 1)
          v = sh.Dd[t] * lrow[t] + sh.Do[t] * lrow[t + 1];
        else
          v = sh.Do[t - 1] * lrow[t - 1] + sh.Dd[t] * lrow[t];
      }
      sh.w[t] = v;
    }
  };
  // record a 1x1 pivot d in column col (this CTA's rows) and in D
  auto finish_1x1 = [&](int p, double d, const double* col) {
    if (d > 0)
      ++n_pos;
    else if (d < 0)
      ++n_neg;
    else
      ++n_zero;
    thread_rmax = fmax(thread_rmax, fabs(d));
    const double inv = 1.0 / d;
    for (int i = max(base, k + 1) + threadIdx.x; i < rend; i += kCT) {
      const int li = i - base;
      const double a = col[li];
      thread_rmax = fmax(thread_rmax, fabs(a));
      const double l = a * inv;
      Lr[p * R + li] = l;
      F[k * ld + i] = l;
    }
    if (threadIdx.x == 0) {
      sh.Dd[p] = d;
      sh.Do[p] = 0.0;
      sh.pk[p] = 0;
    }
    if (q == 0 && threadIdx.x == 0) {
      F[k * ld + k] = d;
      f.Dd[k] = d;
      f.Do[k] = 0.0;
      f.pk[k] = 0;
    }
  };

  // ---- the panel: speculative runs of 1x1 pivots at k, verified against
  // lambda after the fact (see the file comment), and one sequential
  // decision at each pivot where a run stopped; a sequential decision that
  // turns out to be a plain 1x1 at k starts the next speculative run (a
  // restart: the panel's earlier pivots enter as a rank-p0 correction of the
  // restart's columns).
  int spec_carry = S.spec;  // consecutive panels whose first speculation failed at its first pivot
  bool try_spec = spec_carry < kSpecRetry;
  bool first_spec = true, spec_tried = false, any_seq = false, any_accept = false;
  int restarts = 0;
  double* lblk = stage;               // restart: L of the block rows for the earlier pivots (np x p0)
  double* wblk = stage + kStageHalf;  // restart: D L(block row, :)^T (np x p0)
  while (k < pe) {
    if (try_spec) {
      try_spec = false;
      spec_tried = true;
      const int k0 = k, p0 = k0 - ps, np = pe - k0;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int r0 = max(base, pe);
      if (!first_spec) ++restarts;
      pf_col = -1;
      // warp 0 stages the raw diagonal block (lower triangle) and factors it
      // as soon as it lands; warps 1.. stage the raw block columns of this
      // CTA's rows below the block into Lr (columns p0 ..) meanwhile
      // rows [s0, e0): the CTA's rows below the block widened to whole
      // 16-byte pairs (the extra slot before r0 and after rend is spare)
      const int s0 = r0 & ~1, e0 = (rend + 1) & ~1;
      const bool have_rows = r0 < rend;
      // static pivoting: expected sign of block row `lane`, loaded now so the
      // diagonal-block chain below reads it from a register
      const int lane_sign = (o.mode == 1 && o.sign_final && warp == 0 && lane < np) ? o.sign_final[f.fidx[k0 + lane]] : 0;
      if (warp == 0) {
        for (int j = 0; j < np; ++j)
          for (int i = j + lane; i < np; i += 32) cp_async8(&sh.db[i][j], F + static_cast<int64_t>(k0 + j) * ld + k0 + i);
        cp_async_commit();
      } else if (threadIdx.x == 32 && have_rows) {
        const uint32_t bytes = static_cast<uint32_t>(e0 - s0) * sizeof(double);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&rows_bar)),
                     "r"(bytes * static_cast<uint32_t>(np))
                     : "memory");
        for (int c = 0; c < np; ++c)
          bulk_copy_g2s(Lr + (p0 + c) * R + (s0 - base), F + static_cast<int64_t>(k0 + c) * ld + s0, bytes, &rows_bar);
      }
      if (p0 > 0) {
        // restart: every CTA receives the L rows of the block from their
        // owners and forms W = D L_blk^T itself (D is replicated)
        const int lo = max(base, k0), hi = min(rend, pe);
        const int cnt = hi > lo ? (hi - lo) * p0 : 0;
        for (int t = threadIdx.x; t < cnt; t += kCT) {
          const int i = lo + t / p0, tt = t % p0;
          const double v = Lr[tt * R + (i - base)];
          for (int dd = 0; dd < CS; ++dd) remote(lblk, dd)[(i - k0) * p0 + tt] = v;
        }
        __threadfence();
        cluster.sync();
        for (int t = threadIdx.x; t < np * p0; t += kCT) {
          const double* lr = lblk + (t / p0) * p0;
          const int tt = t % p0;
          const int kind = sh.pk[tt];
          double v;
          if (kind == 0)
            v = sh.Dd[tt] * lr[tt];
          else if (kind == 1)
            v = sh.Dd[tt] * lr[tt] + sh.Do[tt] * lr[tt + 1];
          else
            v = sh.Do[tt - 1] * lr[tt - 1] + sh.Dd[tt] * lr[tt];
          wblk[t] = v;
        }
      }
      if (p0 > 0) __syncthreads();  // wblk complete before any warp reads it
      if (warp == 0) {
        cp_async_wait_all();
        __syncwarp();
        if (p0 > 0) {
          // current values of the diagonal block: raw - L_blk W^T
          for (int t = lane; t < np * np; t += 32) {
            const int i = t / np, j = t % np;
            if (j <= i) {
              double acc = 0.0;
              for (int tt = 0; tt < p0; ++tt) acc += lblk[i * p0 + tt] * wblk[j * p0 + tt];
              sh.db[i][j] -= acc;
            }
          }
          __syncwarp();
        }
      } else {
        if (have_rows) {
          if (!mbar_wait_bounded(&rows_bar, rows_phase)) {
            atomicCAS(&g->error, 0, kPanelErrTimeout);
            mbar_wait_bounded(&rows_bar, rows_phase);  // the copies must land before the CTA moves on
          }
        }
        if (p0 > 0) {
          // this warp's own staged rows: subtract the earlier pivots, L_row W^T
          for (int c = 0; c < np; ++c)
            for (int i = r0 + threadIdx.x - 32; i < rend; i += kCT - 32) {
              const int li = i - base;
              double acc = 0.0;
              for (int tt = 0; tt < p0; ++tt) acc += Lr[tt * R + li] * wblk[c * p0 + tt];
              Lr[(p0 + c) * R + li] -= acc;
            }
        }
      }
      if (have_rows) rows_phase ^= 1;  // every thread: the barrier's phase of this staging is consumed
      // diagonal block, left-looking: warp 0 of every CTA, lane = row (the
      // row lives in sh.db, conflict-free with the odd row stride). The sums
      // use four partial accumulators to shorten the dependency chain; |a| of
      // the column values go to shared memory and are reduced afterwards.
      if (warp == 0) {
        const double floorv = fmax(o.static_abs_floor, o.static_rel_floor * orig_max);
        const int lr = lane < np ? lane : 0;
        for (int c = 0; c < np; ++c) {
          double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
          int t = 0;
          for (; t + 4 <= c; t += 4) {
            s0 = fma(sh.db[lr][t], sh.wv[c][t], s0);
            s1 = fma(sh.db[lr][t + 1], sh.wv[c][t + 1], s1);
            s2 = fma(sh.db[lr][t + 2], sh.wv[c][t + 2], s2);
            s3 = fma(sh.db[lr][t + 3], sh.wv[c][t + 3], s3);
          }
          for (; t < c; ++t) s0 = fma(sh.db[lr][t], sh.wv[c][t], s0);
          const double a = sh.db[lr][c] - ((s0 + s1) + (s2 + s3));
          const double akk = __shfl_sync(0xffffffffu, a, c);
          double d = akk, applied = 0.0;
          if (o.mode == 1) {
            // static pivoting (dense_kernel.hpp:982-1034), as in the sequential path
            const int sign = __shfl_sync(0xffffffffu, lane_sign, c);
            bool need;
            if (sign > 0)
              need = akk < floorv;
            else if (sign < 0)
              need = akk > -floorv;
            else
              need = fabs(akk) < floorv;
            if (need) {
              const double sg = (sign != 0) ? static_cast<double>(sign) : (akk >= 0.0 ? 1.0 : -1.0);
              d = akk + sg * S.delta;
              applied = d - akk;
            }
          }
          const double inv = __drcp_rn(d);
          __syncwarp();
          if (lane > c && lane < np) {
            const double l = a * inv;
            sh.db[lane][c] = l;
            sh.aabs[c][lane] = fabs(a);
            sh.wv[lane][c] = d * l;
          } else if (lane == c) {
            sh.db[c][c] = d;
          }
          if (lane == 0) {
            sh.dv[c] = d;
            sh.iv[c] = inv;
            sh.pv[c] = applied;
          }
          __syncwarp();
        }
      }
      __syncthreads();
      // lambda and running-max parts of the diagonal-block rows
      if (threadIdx.x < np) {
        const int c = threadIdx.x;
        double lm = 0.0, rv = fabs(sh.dv[c]);
        for (int i = c + 1; i < np; ++i) {
          const double v = sh.aabs[c][i];
          if (k0 + i < effEnd) lm = fmax(lm, v);
          rv = fmax(rv, v);
        }
        sh.lamd[c] = lm;
        sh.rmd[c] = rv;
      }
      // rows below the block, left-looking: the raw block columns of this
      // CTA's rows are in Lr (staged above; a restart first subtracts the
      // earlier pivots, L_row W^T), then each thread takes one row at a time
      // into registers and walks it pivot by pivot, touching only its own
      // rows, so no synchronisation is needed between pivots; the L(c, t) are
      // warp-uniform (broadcast) shared loads. Lr receives the current values
      // a_ic = raw_ic - sum_t a_it L_ct (L = a_ic / d_c on write-back). Columns
      // past np compute unused values (column c depends on columns t < c only).
      for (int i = r0 + threadIdx.x; i < rend; i += kCT) {
        const int li = i - base;
        double a[kSpecMax];
#pragma unroll
        for (int c = 0; c < kSpecMax; ++c) a[c] = (c < np) ? Lr[(p0 + c) * R + li] : 0.0;
#pragma unroll
        for (int c = 1; c < kSpecMax; ++c) {
          // sum_t L_it d_t L_ct = sum_t a_it L_ct (a_it = L_it d_t): even and
          // odd t in two partial sums
          double s0 = 0.0, s1 = 0.0;
#pragma unroll
          for (int t = 0; t < c; ++t) {
            if (t & 1)
              s1 = fma(a[t], sh.db[c][t], s1);
            else
              s0 = fma(a[t], sh.db[c][t], s0);
          }
          a[c] -= s0 + s1;
          asm volatile("" ::: "memory");  // keep the next pivot's loads from being hoisted (registers)
        }
#pragma unroll
        for (int c = 0; c < kSpecMax; ++c)
          if (c < np) Lr[(p0 + c) * R + li] = a[c];
      }
      __syncthreads();
      // per pivot and warp: lambda part (eligible rows) and running-max part
      // (all rows) of this CTA's rows below the block
      for (int c = warp; c < np; c += kCT / 32) {
        double lm = 0.0, rv = 0.0;
        for (int i = r0 + lane; i < rend; i += 32) {
          const double v = fabs(Lr[(p0 + c) * R + (i - base)]);
          if (i < effEnd) lm = fmax(lm, v);
          rv = fmax(rv, v);
        }
        lm = warp_max_nonneg(lm);
        rv = warp_max_nonneg(rv);
        if (lane == 0) {
          sh.lamw[0][c] = lm;
          sh.rvw[0][c] = rv;
        }
      }
      __syncthreads();
      int kstar = np;
      if (o.mode != 1) {
        // lambda per pivot: this CTA's part to every CTA of the cluster
        if (threadIdx.x < np) {
          const double lc = sh.lamw[0][threadIdx.x];
          for (int dd = 0; dd < CS; ++dd) *cluster.map_shared_rank(&sh.lamx[q][threadIdx.x], dd) = lc;
        }
        cluster.sync();
        if (warp == 0) {
          // the sequential path's 1x1-at-k decision (dense_kernel.hpp:576-600),
          // one lane per pivot; the first failing pivot ends the accepted prefix
          bool fail = false;
          if (lane < np) {
            const double isolatedFloor = fmax(o.zero_tol, o.rel_floor * orig_max);
            double lam = sh.lamd[lane];
            for (int dd = 0; dd < CS; ++dd) lam = fmax(lam, sh.lamx[dd][lane]);
            const double akk = sh.dv[lane];
            const bool pass = (lam <= o.zero_tol) ? (fabs(akk) > isolatedFloor) : (fabs(akk) >= kAlphaBK * lam);
            fail = !pass;
          }
          const unsigned bad = __ballot_sync(0xffffffffu, fail);
          if (lane == 0) sh.kstar = bad ? __ffs(bad) - 1 : np;
        }
        __syncthreads();
        kstar = sh.kstar;
      }
      if (first_spec) spec_carry = kstar > 0 ? 0 : spec_carry + 1;
      first_spec = false;
      if (kstar > 0) {
        any_accept = true;
        for (int c = 0; c < kstar; ++c) {
          const double iv = sh.iv[c];
          for (int i = r0 + threadIdx.x; i < rend; i += kCT)
            F[static_cast<int64_t>(k0 + c) * ld + i] = Lr[(p0 + c) * R + (i - base)] * iv;
        }
        if (q == 0) {
          for (int c = 0; c < kstar; ++c)
            for (int i = c + threadIdx.x; i < np; i += kCT) F[static_cast<int64_t>(k0 + c) * ld + k0 + i] = sh.db[i][c];
          for (int c = threadIdx.x; c < kstar; c += kCT) {
            f.Dd[k0 + c] = sh.dv[c];
            f.Do[k0 + c] = 0.0;
            f.pk[k0 + c] = 0;
          }
        }
        // inertia of the accepted pivots (only thread 0's counters are
        // written back): one ballot each over warp 0's lanes; the
        // perturbations (static mode) are summed in pivot order
        if (warp == 0) {
          const bool in = lane < kstar;
          const double d = in ? sh.dv[lane] : 0.0;
          const unsigned pos = __ballot_sync(0xffffffffu, in && d > 0);
          const unsigned neg = __ballot_sync(0xffffffffu, in && d < 0);
          const unsigned zer = __ballot_sync(0xffffffffu, in && !(d > 0) && !(d < 0));
          const unsigned per = __ballot_sync(0xffffffffu, in && sh.pv[lane] != 0.0);
          if (lane == 0) {
            n_pos += __popc(pos);
            n_neg += __popc(neg);
            n_zero += __popc(zer);
            if (per)
              for (int c = 0; c < kstar; ++c)
                if (sh.pv[c] != 0.0) {
                  pert += fabs(sh.pv[c]);
                  ++nPert;
                }
          }
        }
        if (threadIdx.x < kstar) {
          // running max of the accepted columns (one thread per column)
          thread_rmax = fmax(thread_rmax, fmax(sh.rmd[threadIdx.x], sh.rvw[0][threadIdx.x]));
        }
        k = k0 + kstar;
        if (k < pe) {
          // The sequential decision at k needs, for the accepted pivots: L
          // of this CTA's rows in Lr (below the block: a / d as written to F;
          // block rows: sh.db), D in sh.Dd/Do/pk, and w = D L(k, :)^T (the
          // earlier pivots' part from wblk, the run's part from sh.wv).
          for (int c = 0; c < kstar; ++c) {
            const double iv = sh.iv[c];
            for (int i = r0 + threadIdx.x; i < rend; i += kCT) Lr[(p0 + c) * R + (i - base)] *= iv;
            for (int i = max(base, k0 + c + 1) + threadIdx.x; i < min(rend, pe); i += kCT)
              Lr[(p0 + c) * R + (i - base)] = sh.db[i - k0][c];
          }
          if (threadIdx.x < kstar) {
            sh.Dd[p0 + threadIdx.x] = sh.dv[threadIdx.x];
            sh.Do[p0 + threadIdx.x] = 0.0;
            sh.pk[p0 + threadIdx.x] = 0;
            sh.w[p0 + threadIdx.x] = sh.wv[kstar][threadIdx.x];
          }
          for (int t = threadIdx.x; t < p0; t += kCT) sh.w[t] = wblk[kstar * p0 + t];
          __syncthreads();
        }
      }
      if (k >= pe) break;
    }
    any_seq = true;
    const int p = k - ps;
    const int b = step & 1;
    ++step;
    current_column_pf(k, k, p, sh.w, vk);
    __syncthreads();
    // fast-path exchange: partial argmax (threshold) and the values every
    // CTA needs to continue without a second barrier
    ArgMax am{0.0, -1};
    if (o.mode != 1) {
      for (int i = max(base, k + 1) + threadIdx.x; i < min(rend, effEnd); i += kCT)
        am = argmax_combine(am, ArgMax{fabs(vk[i - base]), i});
      am = block_argmax<kCT>(am, sh.red_v, sh.red_i);
    }
    const bool haveNext = (k + 1 < pe) && (k + 1 < m);
    const int o1 = haveNext ? owner(k + 1) : -1;
    // one thread per destination CTA
    if (threadIdx.x < CS) {
      const int dd = threadIdx.x;
      remote(sh.fx_v[b], dd)[q] = am.v;
      remote(sh.fx_i[b], dd)[q] = am.i;
      if (q == owner(k)) {
        remote(sh.fx_kk, dd)[b] = vk[k - base];
        remote(sh.fx_sign, dd)[b] = (o.mode == 1 && o.sign_final) ? o.sign_final[f.fidx[k]] : 0;
      }
      if (q == o1) remote(sh.fx_k1, dd)[b] = vk[k + 1 - base];
    }
    if (q == o1)
      for (int t = threadIdx.x; t < p * CS; t += kCT)
        remote(sh.fx_row[b], t / p)[t % p] = Lr[(t % p) * R + (k + 1 - base)];
    // prefetch the next column while the exchange completes
    if (haveNext) prefetch(k + 1, k + 1);
    // the cluster barrier orders the distributed shared-memory stores; the
    // global stores of this step are not read by other CTAs in this launch
    cluster.sync();
    const double akk = sh.fx_kk[b];

    if (o.mode == 1) {
      // static pivoting (dense_kernel.hpp:982-1034), decided by every CTA
      const int sign = sh.fx_sign[b];
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
      finish_1x1(p, d, vk);
      if (haveNext) local_w_next(p, d, sh.fx_row[b], sh.fx_k1[b]);
      __syncthreads();
      ++k;
      try_spec = true;
      continue;
    }

    ArgMax gm{sh.fx_v[b][0], sh.fx_i[b][0]};
    for (int dd = 1; dd < CS; ++dd) gm = argmax_combine(gm, ArgMax{sh.fx_v[b][dd], sh.fx_i[b][dd]});
    const double lambda = gm.v;
    const int r = gm.i;
    int dec;
    int dec_kind = 0;  // the seq_dec slot of this decision
    double arr = 0.0, vkr = 0.0;
    if (lambda <= o.zero_tol) {
      const double isolatedFloor = fmax(o.zero_tol, o.rel_floor * orig_max);
      dec = (fabs(akk) <= isolatedFloor) ? 3 : 0;
    } else if (fabs(akk) >= kAlphaBK * lambda) {
      dec = 0;
    } else if (r >= S.ob_end && ps > S.ob) {
      // the partner lies beyond the outer block while earlier panels of the
      // block have not been applied there yet: stop before pivot k so the
      // deferred update is applied first, then restart the block at k
      dec = 4;
    } else {
      // partner column r (slow path)
      if (q == owner(r)) {
        d_times_row(r, p, sh.rowtmp);
        __syncthreads();
        for (int t = threadIdx.x; t < p * CS; t += kCT) remote(sh.wr, t / p)[t % p] = sh.rowtmp[t % p];
      }
      __threadfence();
      cluster.sync();
      current_column(r, k, p, sh.wr, vr);
      double smx = 0.0;
      for (int i = max(base, k) + threadIdx.x; i < min(rend, effEnd); i += kCT)
        if (i != r) smx = fmax(smx, fabs(vr[i - base]));
      smx = block_max<kCT>(smx, sh.red_v);
      if (threadIdx.x == 0) {
        for (int dd = 0; dd < CS; ++dd) remote(sh.ex_v, dd)[q] = smx;
        if (q == owner(r))
          for (int dd = 0; dd < CS; ++dd) {
            double* x = remote(sh.ex_x, dd);
            x[1] = vr[r - base];
            x[2] = vk[r - base];
          }
      }
      __threadfence();
      cluster.sync();
      double sigma = 0.0;
      for (int dd = 0; dd < CS; ++dd) sigma = fmax(sigma, sh.ex_v[dd]);
      arr = sh.ex_x[1];
      vkr = sh.ex_x[2];
      if (fabs(akk) * sigma >= kAlphaBK * lambda * lambda)
        dec = 0;
      else if (fabs(arr) >= kAlphaBK * sigma)
        dec = 1;
      else
        dec = 2;
      dec_kind = dec + 1;
      // the slow path consumed extra barriers; make every CTA finish reading
      // the exchange slots before anyone writes them again
      cluster.sync();
    }
    if (q == 0 && threadIdx.x == 0 && dec <= 2) atomicAdd(&g->seq_dec[dec_kind], 1);
    if (dec == 3) {
      stopped = true;
      break;
    }
    if (dec == 4) {
      flush = true;
      break;
    }
    if (dec == 0) {
      finish_1x1(p, akk, vk);
      if (haveNext) local_w_next(p, akk, sh.fx_row[b], sh.fx_k1[b]);
      __syncthreads();
      k += 1;
      // a plain 1x1 at k by the first test: the next pivots likely are too
      try_spec = dec_kind == 0;
      continue;
    }
    pf_col = -1;  // an interchange invalidates the prefetched column
    if (dec == 1) {
      interchange(k, r, true);
      finish_1x1(p, arr, vr);
      __syncthreads();
      k += 1;
    } else {
      // 2x2 at (k, r): bring r to k+1
      if (r != k + 1) interchange(k + 1, r, true);
      const double d11 = akk, d21 = vkr, d22 = arr;
      const double det = d11 * d22 - d21 * d21;
      // cluster-uniform value (the running max known at panel start), so
      // every thread takes the same branch
      const double rm1 = fmax(1.0, rm_known);
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
      for (int i = max(base, k + 2) + threadIdx.x; i < rend; i += kCT) {
        const int li = i - base;
        const double a0 = vk[li], a1 = vr[li];
        thread_rmax = fmax(thread_rmax, fmax(fabs(a0), fabs(a1)));
        const double l0 = a0 * inv11 + a1 * inv21;
        const double l1 = a0 * inv21 + a1 * inv22;
        Lr[p * R + li] = l0;
        Lr[(p + 1) * R + li] = l1;
        F[k * ld + i] = l0;
        F[(k + 1) * ld + i] = l1;
      }
      if (threadIdx.x == 0) {
        sh.Dd[p] = d11;
        sh.Dd[p + 1] = d22;
        sh.Do[p] = d21;
        sh.Do[p + 1] = 0.0;
        sh.pk[p] = 1;
        sh.pk[p + 1] = 2;
      }
      if (q == 0 && threadIdx.x == 0) {
        F[k * ld + k] = d11;
        F[k * ld + k + 1] = d21;
        F[(k + 1) * ld + k + 1] = d22;
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
    // after an interchange or a 2x2 the next row's w comes from its owner
    if (k < pe) {
      const int pn = k - ps;
      if (q == owner(k)) {
        d_times_row(k, pn, sh.rowtmp);
        __syncthreads();
        for (int t = threadIdx.x; t < pn * CS; t += kCT) remote(sh.w, t / pn)[t % pn] = sh.rowtmp[t % pn];
      }
      __threadfence();
      cluster.sync();
    }
  }

  // ---- finish: running max by a global atomic (monotone), state by rank 0
  const double lmax = block_max<kCT>(thread_rmax, sh.red_v);
  if (threadIdx.x == 0) atomic_max_nonneg(&st[s].running_max, lmax);
  const bool done = stopped || k >= effEnd;
  if (done)
    for (int t = q * kCT + threadIdx.x; t < m; t += CS * kCT) f.lpos[f.lperm[t]] = t;
  if (q == 0 && threadIdx.x == 0) {
    FrontState& W = st[s];
    W.orig_max = orig_max;
    W.delta = S.delta;
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
    W.far = (done || flush || k >= S.ob_end) ? 1 : 0;
    W.spec = spec_carry < kSpecRetry ? spec_carry : kSpecRetry;
    int* counter = !spec_tried ? &g->seq_panels
                   : !any_seq  ? &g->spec_full
                   : any_accept ? &g->spec_partial
                                : &g->spec_failed;
    atomicAdd(counter, 1);
    if (restarts) atomicAdd(&g->spec_restarts, restarts);
    int flags = flush ? kFlagFlush : 0;
    if (done) {
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
  cluster.sync();
}

// Rows per CTA slot of the cluster panel's shared arrays: the rows a CTA
// holds, plus a spare slot at each end of a column for the 16-byte widened
// bulk copies, rounded to even.
int cluster_rows(int max_m, int cs) { return (((max_m + cs - 1) / cs) + 2 + 1) & ~1; }

size_t cluster_panel_smem(int max_m, int nb, int cs) {
  const int R = cluster_rows(max_m, cs);
  return (2 + static_cast<size_t>(nb + 4) * R + 2 * kStageHalf) * sizeof(double);
}

bool cluster_size_fits(int max_m, int cs, int nb) {
  const size_t limit = 184 * 1024;  // + the static ClusterShared (~38 KB) <= 227 KB
  return (cs == 2 || cs == 4 || cs == 8 || cs == 16) && nb >= 1 && nb <= kNBMax - 2 &&
         cluster_panel_smem(max_m, nb, cs) <= limit;
}

int panel_width_for(int max_m, int count) {
  if (cluster_size_for(max_m, count, kPanelWidth) > 0) return kPanelWidth;
  for (int nb = kPanelWidth - 4; nb >= 8; nb -= 4)
    if (cluster_size_fits(max_m, 16, nb)) return nb;
  return kPanelWidth;
}

int cluster_size_for(int max_m, int count, int nb) {
  // The panel is latency-bound: a CTA costs a fixed ~8 us (the diagonal
  // block's pivot chain, the exchanges) plus ~10 ns per row it holds, and
  // one CTA runs per SM (200 registers x 256 threads). More CTAs per front
  // shorten each CTA; fewer let more fronts run in one wave. Pick the
  // cluster size with the smallest modelled time (waves x CTA time).
  int best = 0;
  double best_t = 0.0;
  for (int cs : {2, 4, 8, 16}) {
    if (!cluster_size_fits(max_m, cs, nb)) continue;
    const double waves = std::ceil(static_cast<double>(count) * cs / 148.0);
    const double t = waves * (8.0 + 0.01 * ((max_m + cs - 1) / cs));
    if (best == 0 || t < best_t) {
      best = cs;
      best_t = t;
    }
  }
  return best;  // 0: too large for the cluster kernel
}

cudaError_t configure_cluster_panel() {
  cudaError_t e = cudaFuncSetAttribute(cluster_panel_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 184 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_panel_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 184 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_panel_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 184 * 1024);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(cluster_panel_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 184 * 1024);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(cluster_panel_kernel<16>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

cudaError_t launch_cluster_panel(const FrontDesc* fronts, FrontState* st, const int* list, int count, int max_m,
                                 int nb, const KernelOpts& o, FactorGlobals* g, int level, int dynamic,
                                 cudaStream_t stream, int cs_choice) {
  if (count <= 0) return cudaSuccess;
  const int cs = cluster_size_fits(max_m, cs_choice, nb) ? cs_choice : cluster_size_for(max_m, count, nb);
  if (cs == 0) return cudaErrorInvalidValue;
  const int R = cluster_rows(max_m, cs);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs * count);
  cfg.blockDim = dim3(kCT);
  cfg.dynamicSmemBytes = cluster_panel_smem(max_m, nb, cs);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  switch (cs) {
    case 16:
      return cudaLaunchKernelEx(&cfg, cluster_panel_kernel<16>, fronts, st, list, nb, R, o, g, level, dynamic);
    case 8:
      return cudaLaunchKernelEx(&cfg, cluster_panel_kernel<8>, fronts, st, list, nb, R, o, g, level, dynamic);
    case 4:
      return cudaLaunchKernelEx(&cfg, cluster_panel_kernel<4>, fronts, st, list, nb, R, o, g, level, dynamic);
    default:
      return cudaLaunchKernelEx(&cfg, cluster_panel_kernel<2>, fronts, st, list, nb, R, o, g, level, dynamic);
  }
}

}  // namespace symla_gpu
