// Mixed-precision far (outer-block) Schur-complement update on the 5th-gen
// tensor cores: tcgen05.mma kind::tf32 with the accumulator in TMEM and the
// operands staged by TMA.
//
//   C(i, j) -= sum_q L(i, q) W(j, q),   W = L D,   i >= j,
//   i, j in [c0, m), q in [ob, k1)   (the deferred pivots of the block)
//
// Precision: every FP64 operand x is split into two TF32 parts,
// x ~ hi + lo with hi = tf32(x) and lo = tf32(x - hi) (about 22 significant
// bits together), and the product uses three MMAs, hi*hi + hi*lo + lo*hi,
// accumulated in FP32 in TMEM; the FP64 front is then updated with the
// FP32 result. TF32 keeps FP32's exponent range, so no block scaling is
// needed for range; pivots, D, the near (in-block) updates, L and the
// refinement residual stay FP64. The reference evaluates the same update in
// FP64 (dense_kernel.hpp:806-821); iterative refinement against the true
// matrix recovers full accuracy.
//
// Pipeline per 128 x 128 output tile: a pre-pass writes hi/lo planes of L
// and W for rows [c0, m) into a workspace (row-major, 4 planes of KPAD
// floats per row); TMA loads 32-column boxes (128 B rows, 128B swizzle) of
// the A (rows i) and B (rows j) planes into a 2-stage shared-memory ring;
// one thread issues the MMAs and commits them to mbarriers; the four warps
// then read the accumulator with tcgen05.ld and subtract it from C. Every
// mbarrier wait is bounded in time: on timeout the kernel records an error,
// waits (again bounded) for what it has in flight and frees its TMEM.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "factor_kernels.h"
#include "reduce.cuh"

namespace symla_gpu {

namespace {

constexpr int kTM = 128;       // tile rows (UMMA M)
constexpr int kTN = 128;       // tile columns (UMMA N)
constexpr int kBoxK = 32;      // floats per TMA box row (128 B)
constexpr int kThreads = 128;  // 4 warps: one per 32-lane TMEM quarter
constexpr int kStageBytes = 4 * kTM * kBoxK * 4;  // A_hi, A_lo, B_hi, B_lo
constexpr int kStages = 2;
constexpr int kMaxFronts = 512;
constexpr int kSplitRows = 8;   // rows per pass of the split pre-pass (4 x 8 x (kTcKpad + 1) floats of static shared memory)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Non-blocking probe of phase completion (test_wait never suspends, so a
// spin over it is bounded by the clock check in mbar_wait).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait; false on timeout, with the timeout bit set in the error word
// when err is given. The wait ends once limit_ns of the global timer have
// passed or after limit_ns / 8 unsuccessful probes (a probe takes longer than
// 8 ns), whichever comes first: a limit below the timer's resolution still
// ends the wait. Gives up early once another CTA recorded an error.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint64_t limit_ns) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  const uint64_t max_probes = limit_ns / 8;
  for (uint64_t it = 1;; ++it) {
    if (it > max_probes || ((it & 15) == 0 && global_ns() - t0 > limit_ns)) {
      if (err) atomicOr(err, kTcErrTimeout);
      return false;
    }
    if (mbar_test(bar, parity)) return true;
    if ((it & 63) == 0 && err && *reinterpret_cast<volatile int*>(err) != 0) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// K-major operand in shared memory, 128-byte swizzle (8-row atoms of
// 1024 B): start address, leading offset 1 (unused with swizzle), stride
// offset 1024 B between 8-row groups, descriptor version 1, layout 2.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>(1024 >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(2) << 61;
  return d;
}

// kind::tf32, D = F32, A = B = TF32, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kTN >> 3) << 17) | ((kTM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ bool far_range(const FrontState& S, int m, int& c0, int& q0, int& q1) {
  if (!S.far) return false;
  q0 = S.ob;
  q1 = S.k;
  c0 = max(S.ob_end, S.k);
  return q1 > q0 && m > c0;
}

__device__ __forceinline__ int tc_tiles(int m, int c0) {
  int n = 0;
  for (int j = c0; j < m; j += kTN) n += (m - j + kTM - 1) / kTM;
  return n;
}

}  // namespace

// ---------------------------------------------------------------------------
// Pre-pass: hi/lo TF32 planes of L and W = L D for rows [c0, m) and pivots
// [ob, k1) of every front with a far update due. Workspace row i of front s:
// ws[s] + i * 4 * KPAD floats = {L_hi, L_lo, W_hi, W_lo} x KPAD, zero past K.
// Also records max|L| and max|L D| of the block in guard[2 fi], guard[2 fi + 1]
// (zeroed before the launch) for the growth guard tc_block_ok.
__global__ void __launch_bounds__(256) tc_split_kernel(const FrontDesc* __restrict__ fronts,
                                                       const FrontState* __restrict__ st,
                                                       const int* __restrict__ list, int count,
                                                       float* const* __restrict__ ws, double* guard,
                                                       const FactorGlobals* g, int level, int dynamic) {
  if (level_skipped(g, level, dynamic)) return;
  __shared__ float tile[4][kSplitRows][kTcKpad + 1];
  __shared__ double red[8];
  const int fi = blockIdx.y;
  if (fi >= count) return;
  const int s = list[fi];
  const FrontDesc f = fronts[s];
  const FrontState S = st[s];
  int c0, q0, q1;
  if (!far_range(S, f.m, c0, q0, q1)) return;
  const int K = q1 - q0;
  if (K > kTcKpad) return;  // wider than the workspace: tc_block_ok sends it to the FP64 update
  double lmax = 0.0, wmax = 0.0;
  const int64_t ld = f.ld;
  float* w = ws[fi];
  for (int r0 = c0 + blockIdx.x * kSplitRows; r0 < f.m; r0 += gridDim.x * kSplitRows) {
    const int nr = min(kSplitRows, f.m - r0);
    // reads: consecutive threads take consecutive rows of one pivot column
    for (int t = threadIdx.x; t < kSplitRows * kTcKpad; t += 256) {
      const int rr = t % kSplitRows, q = t / kSplitRows;
      float lh = 0.f, ll = 0.f, wh = 0.f, wl = 0.f;
      if (rr < nr && q < K) {
        const int i = r0 + rr, pq = q0 + q;
        const double l = f.F[pq * ld + i];
        const int8_t kind = f.pk[pq];
        double wv = f.Dd[pq] * l;
        if (kind == 1) wv += f.Do[pq] * f.F[(pq + 1) * ld + i];
        if (kind == 2) wv += f.Do[pq - 1] * f.F[(pq - 1) * ld + i];
        lmax = fmax(lmax, fabs(l));
        wmax = fmax(wmax, fabs(wv));
        lh = tf32_rna(static_cast<float>(l));
        ll = tf32_rna(static_cast<float>(l - static_cast<double>(lh)));
        wh = tf32_rna(static_cast<float>(wv));
        wl = tf32_rna(static_cast<float>(wv - static_cast<double>(wh)));
      }
      tile[0][rr][q] = lh;
      tile[1][rr][q] = ll;
      tile[2][rr][q] = wh;
      tile[3][rr][q] = wl;
    }
    __syncthreads();
    // writes: consecutive threads take consecutive floats of a workspace row
    for (int t = threadIdx.x; t < nr * 4 * kTcKpad; t += 256) {
      const int rr = t / (4 * kTcKpad), c = t % (4 * kTcKpad);
      w[static_cast<int64_t>(r0 + rr) * 4 * kTcKpad + c] = tile[c / kTcKpad][rr][c % kTcKpad];
    }
    __syncthreads();
  }
  lmax = block_max<256>(lmax, red);
  wmax = block_max<256>(wmax, red);
  if (threadIdx.x == 0) {
    atomic_max_nonneg(&guard[2 * fi], lmax);
    atomic_max_nonneg(&guard[2 * fi + 1], wmax);
  }
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1) tc_far_update_kernel(const FrontDesc* __restrict__ fronts,
                                                                     FrontState* st, const int* __restrict__ list,
                                                                     int count, const CUtensorMap* __restrict__ maps,
                                                                     const double* __restrict__ guard,
                                                                     FactorGlobals* g, int level, int dynamic,
                                                                     int* err) {
  if (level_skipped(g, level, dynamic)) return;
  const uint64_t wait_ns = g->wait_ns;
  extern __shared__ __align__(1024) unsigned char tsm_raw[];
  // 1024-byte aligned stage ring (128B swizzle atoms)
  unsigned char* ring =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tsm_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], done_bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int tile_end[kMaxFronts];
  __shared__ int s_abort;

  // per-front tile counts (one tile space over every front of the launch)
  for (int t = threadIdx.x; t < count; t += kThreads) {
    const int sf = list[t];
    int c0, q0, q1;
    const FrontState S = st[sf];
    const bool use = far_range(S, fronts[sf].m, c0, q0, q1) &&
                     tc_block_ok(q1 - q0, guard[2 * t], guard[2 * t + 1], g->amax);
    tile_end[t] = use ? tc_tiles(fronts[sf].m, c0) : 0;
    if (blockIdx.x == 0 && tile_end[t] > 0) {
      const double mm = fronts[sf].m, nc = mm - c0;
      const double entries = nc * mm - (static_cast<double>(c0) + mm - 1) * nc / 2.0;
      atomicAdd(&g->flops_far, 2.0 * (q1 - q0) * entries);
    }
  }
  __shared__ int scan_tot[kThreads / 32];
  block_inclusive_scan<kThreads, kMaxFronts / kThreads>(tile_end, count, scan_tot);
  const int total = count > 0 ? tile_end[count - 1] : 0;
  if (static_cast<int>(blockIdx.x) >= total) return;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    mbar_init(&done_bar, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base_s)),
                 "r"(kTN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  uint32_t full_phase[kStages] = {0, 0}, empty_phase[kStages] = {0, 0}, done_phase = 0;
  int issued[kStages] = {0, 0};   // MMA groups committed to empty_bar[s] not yet waited for
  int loading[kStages] = {0, 0};  // TMA loads into stage s not yet observed complete
  bool ok = true;

  // the CTA's tiles increase: the front entry and its column tile advance
  // from where the previous tile left them
  int fi = 0, tj = 0, tj_first = 0;
  for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
    while (tile >= tile_end[fi]) {
      ++fi;
      tj = 0;
      tj_first = 0;
    }
    const int s = list[fi];
    const FrontDesc f = fronts[s];
    const FrontState S = st[s];
    int c0, q0, q1;
    far_range(S, f.m, c0, q0, q1);
    const int m = f.m;
    const int rel = tile - (fi > 0 ? tile_end[fi - 1] : 0);
    for (;;) {
      const int nr = (m - (c0 + tj * kTN) + kTM - 1) / kTM;
      if (rel < tj_first + nr) break;
      tj_first += nr;
      ++tj;
    }
    const int j0 = c0 + tj * kTN, i0 = j0 + (rel - tj_first) * kTM;
    const int K = q1 - q0;
    const int nchunks = (K + kBoxK - 1) / kBoxK;
    const CUtensorMap* map = maps + fi;

    // the tile's C region into L2 while the operands stream in (the
    // epilogue then reads it from L2): warp w's 32 rows of each column are
    // 256 contiguous bytes; lane l covers columns 4l .. 4l + 3
    {
      const int rb = i0 + warp * 32;
      if (rb < m)
        for (int q = 0; q < 4; ++q) {
          const int gj = j0 + lane * 4 + q;
          if (gj < m && gj <= rb + 31) {
            const double* colp = f.F + static_cast<int64_t>(gj) * f.ld + rb;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(colp));
            if (rb + 16 < m) asm volatile("prefetch.global.L2 [%0];" ::"l"(colp + 16));
          }
        }
    }
    if (threadIdx.x == 0) {
      // producer + MMA issuer: chunk c + 1's copy is in flight while chunk
      // c is waited for and multiplied
      auto issue = [&](int c) -> bool {
        const int st_i = c % kStages;
        if (issued[st_i]) {
          if (!mbar_wait(&empty_bar[st_i], empty_phase[st_i], err, wait_ns)) return false;
          empty_phase[st_i] ^= 1;
          issued[st_i] = 0;
        }
        unsigned char* base = ring + st_i * kStageBytes;
        mbar_expect_tx(&full_bar[st_i], kStageBytes);
        const int xk = c * kBoxK;
        tma_load_2d(base, map, 0 * kTcKpad + xk, i0, &full_bar[st_i]);                       // L_hi rows i
        tma_load_2d(base + 1 * kTM * kBoxK * 4, map, 1 * kTcKpad + xk, i0, &full_bar[st_i]);  // L_lo rows i
        tma_load_2d(base + 2 * kTM * kBoxK * 4, map, 2 * kTcKpad + xk, j0, &full_bar[st_i]);  // W_hi rows j
        tma_load_2d(base + 3 * kTM * kBoxK * 4, map, 3 * kTcKpad + xk, j0, &full_bar[st_i]);  // W_lo rows j
        loading[st_i] = 1;
        return true;
      };
      if (!issue(0)) ok = false;
      for (int c = 0; c < nchunks && ok; ++c) {
        const int st_i = c % kStages;
        if (c + 1 < nchunks && !issue(c + 1)) {
          ok = false;
          break;
        }
        unsigned char* base = ring + st_i * kStageBytes;
        if (!mbar_wait(&full_bar[st_i], full_phase[st_i], err, wait_ns)) {
          ok = false;
          break;
        }
        loading[st_i] = 0;
        full_phase[st_i] ^= 1;
        tc_fence_after();
        const uint32_t a_hi = smem_addr(base), a_lo = smem_addr(base + kTM * kBoxK * 4);
        const uint32_t b_hi = smem_addr(base + 2 * kTM * kBoxK * 4), b_lo = smem_addr(base + 3 * kTM * kBoxK * 4);
        for (int ks = 0; ks < kBoxK / 8; ++ks) {
          const uint32_t off = ks * 32;  // 8 tf32 per MMA along K
          const uint32_t acc0 = (c > 0 || ks > 0) ? 1u : 0u;
          umma_tf32(tmem, umma_desc_sw128(a_hi + off), umma_desc_sw128(b_hi + off), acc0);
          umma_tf32(tmem, umma_desc_sw128(a_hi + off), umma_desc_sw128(b_lo + off), 1u);
          umma_tf32(tmem, umma_desc_sw128(a_lo + off), umma_desc_sw128(b_hi + off), 1u);
        }
        umma_commit(&empty_bar[st_i]);
        issued[st_i] = 1;
      }
      if (ok) umma_commit(&done_bar);
      if (!ok) s_abort = 1;
    }
    __syncthreads();
    if (s_abort) {
      ok = false;
      break;
    }
    // accumulator ready
    if (!mbar_wait(&done_bar, done_phase, err, wait_ns)) {
      ok = false;
      s_abort = 1;
    }
    done_phase ^= 1;
    tc_fence_after();
    __syncthreads();
    if (s_abort) {
      ok = false;
      break;
    }
    // epilogue: warp w owns rows i0 + 32w + lane (TMEM lanes 32w..32w+31)
    const int gi = i0 + warp * 32 + lane;
    const int64_t ld = f.ld;
    double tmax = 0.0;
    for (int cc = 0; cc < kTN; cc += 32) {
      uint32_t r[32];
      tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cc, r);
      // all 32 loads of the chunk before any store (the front pointer may
      // alias as far as the compiler knows, so interleaving would serialise)
      double cv[32];
      double* p0 = f.F + static_cast<int64_t>(j0 + cc) * ld + gi;
#pragma unroll
      for (int jj = 0; jj < 32; ++jj) {
        const int gj = j0 + cc + jj;
        cv[jj] = (gi < m && gj < m && gi >= gj) ? p0[jj * ld] : 0.0;
      }
#pragma unroll
      for (int jj = 0; jj < 32; ++jj) {
        const int gj = j0 + cc + jj;
        if (gi < m && gj < m && gi >= gj) {
          const double v = cv[jj] - static_cast<double>(__uint_as_float(r[jj]));
          p0[jj * ld] = v;
          tmax = fmax(tmax, fabs(v));
        }
      }
    }
    tmax = warp_max(tmax);
    if (lane == 0) atomic_max_nonneg(&st[s].running_max, tmax);
    tc_fence_before();
    __syncthreads();  // TMEM read before the next tile overwrites it
    tc_fence_after();
  }

  // drain: wait (bounded by the default limit, whatever the caller's) for
  // copies and MMA groups still in flight; a drain that runs out is recorded
  // separately, since the tensor memory is then released with work possibly
  // outstanding
  if (threadIdx.x == 0)
    for (int i = 0; i < kStages; ++i) {
      bool drained = true;
      if (loading[i]) drained = mbar_wait(&full_bar[i], full_phase[i], nullptr, kDefaultWaitNs) && drained;
      if (issued[i]) drained = mbar_wait(&empty_bar[i], empty_phase[i], nullptr, kDefaultWaitNs) && drained;
      if (!drained) atomicOr(err, kTcErrDrain);
    }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTN));
}

// ---------------------------------------------------------------------------
size_t tc_far_smem() { return static_cast<size_t>(kStages) * kStageBytes + 1024; }

cudaError_t configure_tc_far() {
  return cudaFuncSetAttribute(tc_far_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(tc_far_smem()));
}

void launch_tc_split(const FrontDesc* fronts, const FrontState* st, const int* list, int count, float* const* ws,
                     double* guard, int max_m, const FactorGlobals* g, int level, int dynamic, cudaStream_t stream) {
  if (count <= 0) return;
  const int rows = (max_m + kSplitRows - 1) / kSplitRows;
  const int gx = rows < 128 ? rows : 128;
  tc_split_kernel<<<dim3(gx, count), 256, 0, stream>>>(fronts, st, list, count, ws, guard, g, level, dynamic);
}

void launch_tc_far(const FrontDesc* fronts, FrontState* st, const int* list, int count, const CUtensorMap* maps,
                   const double* guard, int grid, FactorGlobals* g, int level, int dynamic, int* err,
                   cudaStream_t stream) {
  if (count <= 0 || grid <= 0) return;
  tc_far_update_kernel<<<grid, kThreads, tc_far_smem(), stream>>>(fronts, st, list, count, maps, guard, g, level,
                                                                  dynamic, err);
}

int tc_max_fronts() { return kMaxFronts; }

}  // namespace symla_gpu
