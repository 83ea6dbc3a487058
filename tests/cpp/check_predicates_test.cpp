// Host run of the bounds-check predicates of the checked build
// (ma57_b200/csrc/gpu/checked.cuh) on hand-made front tables, good and with
// planted mistakes: every planted mistake must be caught, no good entry
// flagged.
#include <cstdio>
#include <vector>

#include "checked.cuh"

using namespace symla_gpu;

static int failures = 0;
#define EXPECT(cond)                                              \
  do {                                                            \
    if (!(cond)) {                                                \
      std::printf("FAILED line %d: %s\n", __LINE__, #cond);       \
      ++failures;                                                 \
    }                                                             \
  } while (0)

int main() {
  // descriptor shapes: m, ld, ncols, nelig, nextra
  EXPECT(front_shape_ok(10, 10, 3, 3, 0));
  EXPECT(front_shape_ok(10, 10, 3, 5, 2));  // two delayed columns taken over
  EXPECT(front_shape_ok(0, 0, 0, 0, 0));
  EXPECT(!front_shape_ok(10, 9, 3, 3, 0));   // ld < m
  EXPECT(!front_shape_ok(10, 10, 3, 4, 0));  // nelig != ncols + nextra
  EXPECT(!front_shape_ok(4, 4, 3, 5, 2));    // more eligible columns than rows
  EXPECT(!front_shape_ok(-1, 0, 0, 0, 0));

  // storage: a 6 x 6 front (ld 6) inside a 100-double arena
  std::vector<double> arena(100);
  const double* lo = arena.data();
  const double* hi = arena.data() + arena.size();
  EXPECT(storage_ok(arena.data(), 6, 6, lo, hi));
  EXPECT(storage_ok(arena.data() + 64, 6, 6, lo, hi));    // ends exactly at the arena's end
  EXPECT(!storage_ok(arena.data() + 65, 6, 6, lo, hi));   // one past
  EXPECT(!storage_ok(arena.data() + 10, 10, 10, lo, hi));
  EXPECT(!storage_ok(nullptr, 6, 6, lo, hi));
  EXPECT(storage_ok(nullptr, 0, 0, lo, hi));               // an empty front has no storage

  // A scatter entries of a front with m = 8, 3 own columns, 1 delayed row:
  // positions < 3 are own columns, later ones move down by nextra
  const int m = 8, ncols = 3, nextra = 1;
  const long long nnz = 20;
  EXPECT(a_entry_ok(0, 0, 0, ncols, nextra, m, nnz));    // diagonal
  EXPECT(a_entry_ok(1, 6, 19, ncols, nextra, m, nnz));   // pos 6 -> row 7, the last
  EXPECT(!a_entry_ok(1, 7, 0, ncols, nextra, m, nnz));   // pos 7 -> row 8 = m
  EXPECT(!a_entry_ok(2, 1, 0, ncols, nextra, m, nnz));   // above the diagonal
  EXPECT(!a_entry_ok(3, 5, 0, ncols, nextra, m, nnz));   // not an own column
  EXPECT(!a_entry_ok(0, 4, 20, ncols, nextra, m, nnz));  // value index past A
  EXPECT(!a_entry_ok(0, -1, 0, ncols, nextra, m, nnz));

  // extend-add maps of a child with a 4-row contribution block into a
  // 6-row parent: invmap entries in [-1, 4), relmap entries in [0, 6)
  const int invmap[6] = {-1, 0, 1, -1, 2, 3};
  const int relmap[4] = {1, 2, 4, 5};
  for (int v : invmap) EXPECT(in_range(v, -1, 4));
  for (int v : relmap) EXPECT(in_range(v, 0, 6));
  const int bad_inv[2] = {4, -2}, bad_rel[2] = {6, -1};
  for (int v : bad_inv) EXPECT(!in_range(v, -1, 4));
  for (int v : bad_rel) EXPECT(!in_range(v, 0, 6));

  if (failures) return 1;
  std::printf("check_predicates OK\n");
  return 0;
}
