// Bounds checks of the SYMLA_GPU_CHECKED build.
//
// compute-sanitizer cannot be used on the target machines, so the library can
// be built a second time (libsymla_b200_checked.so, -DSYMLA_GPU_CHECKED) in
// which every access whose index comes from a table rather than from a loop
// bound is checked before it is made: the front descriptors and their storage,
// the extend-add maps, the scatter map of A's values, the row indices the
// solves gather and scatter through, and the contribution-block positions the
// assembly reads. A failed check skips the access and records the first
// failure (a code and where it happened) in a status word in device memory;
// nothing traps or asserts. The host reads the word after every factorization
// and solve and turns a failure into SYMLA_ERR_INTERNAL; the context is then
// not used again.
//
// In the ordinary build every check() is the constant true, so the checks
// and the loads that only they need compile away.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace symla_gpu {

enum CheckCode : int {
  kChkNone = 0,
  kChkFrontShape = 1,    // m, ld, ncols, nelig, nextra of a descriptor inconsistent
  kChkFrontStorage = 2,  // a front's m x ld block outside every front allocation
  kChkRowIndex = 3,      // a front row index outside [0, n)
  kChkChildLink = 4,     // a child link's child or contribution-block size out of range
  kChkInvMap = 5,        // parent row -> child contribution-block index out of range
  kChkRelMap = 6,        // child contribution-block index -> parent row out of range
  kChkAEntry = 7,        // A scatter entry outside its front or outside A's values
  kChkPivots = 8,        // a front's pivot count outside [0, nelig]
  kChkGather = 9,        // contribution-block read outside the child's front
  kChkPermute = 10,      // solve permutation entry outside [0, n)
  kChkSolveRow = 11,     // level-solve row index or child workspace row out of range
  kChkWorkspace = 12,    // a front's solve workspace outside the workspace allocation
};

// First failure wins; count keeps counting.
struct CheckWord {
  int count;
  int code;
  long long where;  // the front (or entry) where it happened
};

#ifdef SYMLA_GPU_CHECKED
constexpr bool kCheckedBuild = true;
__device__ __forceinline__ bool check(bool ok, CheckWord* w, int code, long long where) {
  if (!ok && w != nullptr) {
    if (atomicAdd(&w->count, 1) == 0) {
      w->code = code;
      w->where = where;
    }
  }
  return ok;
}
#else
constexpr bool kCheckedBuild = false;
__device__ __forceinline__ bool check(bool, CheckWord*, int, long long) { return true; }
#endif

__host__ __device__ inline bool in_range(long long v, long long lo, long long hi) { return v >= lo && v < hi; }

// A front descriptor's sizes: the eligible columns are its own plus the
// delayed ones it took over, and all of them are among its rows.
__host__ __device__ inline bool front_shape_ok(int m, int ld, int ncols, int nelig, int nextra) {
  return m >= 0 && ld >= m && ncols >= 0 && nextra >= 0 && nelig == ncols + nextra && nelig <= m;
}

// The front's block [F, F + ld * m) inside [lo, hi).
__host__ __device__ inline bool storage_ok(const double* F, int m, int ld, const double* lo, const double* hi) {
  if (m == 0) return true;
  if (F == nullptr || F < lo) return false;
  const long long extent = static_cast<long long>(ld) * m;
  return extent <= static_cast<long long>(hi - F);
}

// One stored entry of A scattered into a front: local column j among the
// front's own columns, pattern position pos (after the delayed rows when it
// is past the own columns) on or below the diagonal, value index inside A.
__host__ __device__ inline bool a_entry_ok(int j, int pos, long long idx, int ncols, int nextra, int m,
                                           long long nnz) {
  if (!in_range(j, 0, ncols) || pos < 0) return false;
  const int i = pos < ncols ? pos : pos + nextra;
  return i >= j && i < m && in_range(idx, 0, nnz);
}

}  // namespace symla_gpu
