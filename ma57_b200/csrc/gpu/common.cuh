// Shared device-side types for the B200 numeric factorize / solve path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "checked.cuh"

namespace symla_gpu {

// One frontal matrix (supernode) as the kernels see it. All pointers are
// device pointers; a front's storage may live in the static arena or, after
// delayed pivots re-planned it, in a per-level allocation.
struct FrontDesc {
  double* F;          // m x m column-major, leading dimension ld; lower triangle authoritative
  int* fidx;          // m final-order row indices (permuted in place by pivoting swaps)
  double* Dd;         // nelig: D diagonal
  double* Do;         // nelig: D(k+1,k) of a 2x2 block starting at k, else 0
  int8_t* pk;         // nelig: 0 = 1x1, 1 = first of 2x2, 2 = second of 2x2
  double* W;          // solve workspace, m x nrhs (column stride wld)
  int* lperm;         // m: pre-pivot local index now at each position (pivoting swaps)
  int* lpos;          // m: inverse of lperm, written when the front is finished
  int m, ld;
  int ncols, nelig, nextra;
  int parent;         // parent front or -1
  int ch_begin, ch_end;  // children, into the ChildLink array
  int a_begin, a_end;    // original-A entries of the own columns
  int level;
  int wld;            // leading dimension of W (>= m)
};

// Child -> parent extend-add maps.
struct ChildLink {
  int child;
  const int* invmap;  // m_parent entries: parent local row -> child CB index, -1 if none
  const int* relmap;  // cb_child entries: child CB index -> parent local row
  int cb;             // contribution block size of the child
};

// Per-front results written by the factor kernels.
struct FrontState {
  int npiv;        // pivots finalized at this front
  int flags;       // bit0 done, bit1 delayed to parent, bit2 leftover at a root (singular)
  int n_pos, n_neg, n_zero;
  int num_perturbed;
  int k;           // next column (panel driver progress)
  int panel_start; // first column of the panel in flight
  int ob, ob_end;  // outer block [ob, ob_end): its pivots' update of the
                   // columns beyond ob_end is deferred to one far update
  int far;         // 1: the far update of [ob, k) is due after this panel
  int spec;        // consecutive panels whose speculative first pivot failed
  double perturb;
  double orig_max;
  double running_max;
  double delta;    // static pivoting delta used for this front
};

enum : int { kFlagDone = 1, kFlagDelayed = 2, kFlagSingularRoot = 4, kFlagFlush = 8 };

// Columns per outer block of the large-front factorization.
constexpr int kOuterBlock = 256;
// Pivots per far update the tensor-core workspace holds (>= kOuterBlock + 1,
// a multiple of 32).
constexpr int kTcKpad = 288;
// Growth guard of the mixed-precision far update. A block of K pivots goes
// to the tensor cores only when max|L| * max|L D| over the rows it updates
// is at most this multiple of max|a_ij| of the original matrix: TF32x3
// rounds each product to about 2^-22 of |l||w|, and that rounding is a
// perturbation of the matrix entry the update lands on (the backward-error
// view of elimination), so it stays a small multiple of 2^-22 max|A|. Blocks
// with larger multipliers (threshold pivoting restricted to the eligible rows
// lets them grow) take the FP64 update instead. Both far-update kernels
// evaluate this one predicate on the same recorded maxima, so each block is
// applied exactly once.
constexpr double kTcGrowthGuard = 8.0;
__host__ __device__ inline bool tc_block_ok(int K, double lmax, double wmax, double amax) {
  return K <= kTcKpad && lmax * wmax <= kTcGrowthGuard * amax;
}

// Error word of the pipelined solve kernels: a wait ran out; (checked build)
// a row index or a child's workspace row was out of range.
constexpr int kSolveErrTimeout = 1;
constexpr int kSolveErrBounds = 8;
// FactorGlobals::error: a panel's bulk staging of its rows did not complete
// within the default wait limit.
constexpr int kPanelErrTimeout = 3;
// FactorGlobals::error: a bulk copy of the FP64 Schur update's staging ring
// did not complete within the default wait limit.
constexpr int kUpdateErrTimeout = 5;
// Error bits of the tensor-core Schur update: a pipeline wait ran out (the
// CTA abandoned its tile), and the drain after such an abandonment could not
// confirm that the CTA's copies and tensor-core operations had finished before
// it released its tensor memory (the context is then not trusted again).
constexpr int kTcErrTimeout = 2;
constexpr int kTcErrDrain = 4;
// Default bound of every device-side wait on another CTA's progress (flags of
// the pipelined solves, mbarriers of the tensor-core update), in ns of the
// global timer; a context may lower it (symla_gpu_set_wait_limit_ns). The
// drain after an abandoned tile always waits up to this default.
constexpr unsigned long long kDefaultWaitNs = 2000000000ull;

// Global counters for one factorization (device, zeroed per call).
struct FactorGlobals {
  int delay_level;     // lowest level that produced a delayed column, or INT_MAX
  int error;           // nonzero: internal error code
  int err_front;
  int unfinished_level;  // graph launches: lowest level left unfinished after its planned iterations
  double flops_near;   // algorithmic flops of the near (in-block) updates
  double flops_far;    // algorithmic flops of the far (deferred) updates
  double amax;         // max |a_ij| of the matrix being factorized (mixed precision only)
  // large-front panels of the last factorization: speculation accepted the
  // whole panel / a prefix / failed at its first pivot; whole sequential panels
  int spec_full, spec_partial, spec_failed, seq_panels;
  unsigned long long wait_ns;  // bound of the tensor-core update's waits (set per call)
  // decisions of the panels' sequential (per-pivot) path: 1x1 at k by the
  // first Bunch-Kaufman test (or an isolated column), 1x1 at k by the sigma
  // test, interchange then 1x1, 2x2
  int seq_dec[4];
  int spec_restarts;  // speculative runs started after a sequential decision inside a panel
};

// Kernels of a level return at once when an earlier level stopped the
// planned (static) pass: a delayed pivot (delay_level) or, in a graph
// launch, a level whose planned panel iterations did not finish it
// (unfinished_level). The host then continues from there.
__device__ __forceinline__ bool level_skipped(const FactorGlobals* g, int level, int dynamic) {
  return !dynamic && min(g->delay_level, g->unfinished_level) < level;
}

// Options visible to kernels.
struct KernelOpts {
  int mode;            // 0 threshold, 1 static
  int precision;       // 0 fp64, 1 mixed
  double zero_tol;
  double rel_floor;
  double static_delta;
  double static_rel_floor;
  double static_abs_floor;
  const int* sign_final;        // n, expected sign in final order (static mode) or nullptr
  const double* front_delta;    // per front delta override or nullptr
  const double* values;         // A values (device), CSC order
  const int* a_j;               // A entry: local column
  const int* a_pos;             // A entry: rowPattern position
  const int* a_idx;             // A entry: index into values
  long long nnz;                // number of A values
  CheckWord* chk;               // status word of the bounds checks (checked build)
};

}  // namespace symla_gpu
