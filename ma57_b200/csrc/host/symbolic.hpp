// Host-side symbolic analysis: fill-reducing ordering, elimination tree,
// column counts, fundamental supernodes and relaxed amalgamation.
//
// This is the analysis that the numeric GPU factorization consumes. It is a
// restatement of the reference's host symbolic pipeline and must produce the
// identical permutation / etree / supernode partition for a given ordering:
//   ordering.hpp:44-75      symmetric pattern of A + A^T without diagonal
//   ordering.hpp:84-149     computeOrdering (AMD / METIS / Natural)
//   elimination_tree.hpp:62-138  Liu etree + explicit row-pattern column counts
//   symbolic.hpp:85-105     postorder (children in increasing index order)
//   symbolic.hpp:195-399    SymbolicFactor::analyze
//
// Only the pattern is used; values are never read here.
#pragma once

#include <cstdint>
#include <vector>

namespace symla_host {

// MetisIperm is the reference's own METIS convention (ordering.hpp:130-141):
// METIS_NodeND's second output array is taken as the pivot order. Metis takes
// the first array, which lists the original vertex at each new position.
enum class OrderingType { AMD = 0, Metis = 1, Natural = 2, MetisIperm = 3 };

// Compressed-column pattern (0-based, square).
struct CscPattern {
  int n = 0;
  std::vector<int> colPtr;  // size n+1
  std::vector<int> rowIdx;  // size nnz
};

// Pattern of A + A^T with the diagonal removed, rows sorted and unique per
// column (ordering.hpp:44-75). `colptr/rowind` may hold either triangle or both.
CscPattern symmetricPatternNoDiag(int n, const int* colptr, const int* rowind);

// Same as above but with every original index i relabelled to newIndexOf[i]
// (equivalent to the reference's permutePatternSymmetric followed by
// buildSymmetricPatternNoDiag, symbolic.hpp:110-134 + elimination_tree.hpp:70).
CscPattern permutedSymmetricPattern(const CscPattern& sym, const std::vector<int>& newIndexOf);

// perm[k] = original index of the k-th pivot.
std::vector<int> computeOrdering(const CscPattern& sym, OrderingType type);

// Approximate minimum degree on the quotient graph (Amestoy, Davis & Duff,
// SIAM J. Matrix Anal. Appl. 17(4), 1996). Input: symmetric pattern without
// diagonal. Output: perm[k] = original index of the k-th pivot.
std::vector<int> amdOrder(const CscPattern& sym);

// Nested dissection through METIS_NodeND (METIS 5 API, 64-bit idx_t as built
// into the CUDA toolkit's libmetis_static.a). Output convention as above;
// with takeIperm the second output array is returned instead (the reference's
// convention, ordering.hpp:130-141).
std::vector<int> metisOrder(const CscPattern& sym, bool takeIperm = false);

struct EliminationTree {
  std::vector<int> parent;    // parent[j] or -1
  std::vector<int> colCount;  // |Struct(L*j)| including the diagonal
  int n = 0;
};

// Liu's etree (union-find with path compression), elimination_tree.hpp:78-96.
std::vector<int> eliminationTreeParent(const CscPattern& permutedSym);

// Postorder of the forest given by parent[] with children visited in
// increasing index order (symbolic.hpp:85-105). Iterative, same visit order.
std::vector<int> postorder(const std::vector<int>& parent);

struct Supernode {
  int firstCol = 0;
  int ncols = 0;
  std::vector<int> rowPattern;  // sorted; first ncols entries are the own columns
  std::int64_t storageNnz() const {
    const std::int64_t m = static_cast<std::int64_t>(rowPattern.size());
    const std::int64_t k = ncols;
    return k * m - k * (k - 1) / 2;
  }
};

// The elimination tree with its column counts (elimination_tree.hpp:62-138)
// from the structures Struct(L*j), which live only until their parent's
// structure is formed. Optionally returns the fundamental supernodes
// (symbolic.hpp:229-247, each with its first column's structure), and fills
// the rowPattern of each of the given contiguous column groups with the
// sorted union of its columns' structures (symbolic.hpp:385-396).
EliminationTree columnStructure(const CscPattern& permutedSym, std::vector<Supernode>* fundamental,
                                std::vector<Supernode>* groups);

struct SymbolicFactorOptions {
  int max_relax_size = 64;
  double max_relax_fill_fraction = 0.25;
};

struct SymbolicFactor {
  std::vector<int> perm;  // final order -> original index
  EliminationTree etree;
  std::vector<Supernode> supernodes;
  std::vector<Supernode> fundamentalSupernodes;
};

// SymbolicFactor::analyze (symbolic.hpp:195-399).
SymbolicFactor analyze(int n, const int* colptr, const int* rowind, OrderingType ordering,
                       const SymbolicFactorOptions& options);

}  // namespace symla_host
