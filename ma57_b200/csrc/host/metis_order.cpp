// Nested-dissection ordering through METIS_NodeND (METIS 5 public API).
//
// The METIS linked here is the static library shipped with the CUDA toolkit
// (libmetis_static.a), built with a 64-bit idx_t: METIS_SetDefaultOptions
// fills METIS_NOPTIONS = 40 eight-byte slots with -1. The reference calls the
// same entry point (ordering.hpp:116-142).
//
// Output convention: perm[k] = original index of the k-th pivot. METIS returns
// two arrays; the first (`perm`) lists, for every position of the reordered
// matrix, the original vertex placed there, which is exactly this convention
// (the separator vertices of the top-level bisection come out last). The
// reference passes METIS's second array (`iperm`) instead; that is the
// inverse permutation, not the nested-dissection order itself. `takeIperm`
// reproduces the reference's choice for callers that need its exact
// permutation.
#include "symbolic.hpp"

#include <cstdint>
#include <stdexcept>
#include <vector>

extern "C" {
int METIS_NodeND(int64_t* nvtxs, int64_t* xadj, int64_t* adjncy, int64_t* vwgt, int64_t* options, int64_t* perm,
                 int64_t* iperm);
}

namespace symla_host {

std::vector<int> metisOrder(const CscPattern& sym, bool takeIperm) {
  const int n = sym.n;
  std::vector<int64_t> xadj(sym.colPtr.begin(), sym.colPtr.end());
  std::vector<int64_t> adjncy(sym.rowIdx.begin(), sym.rowIdx.end());
  if (adjncy.empty()) adjncy.push_back(0);
  std::vector<int64_t> mperm(n), miperm(n);
  int64_t nv = n;
  // Default options (deterministic, fixed seed), 0-based numbering.
  const int status = METIS_NodeND(&nv, xadj.data(), adjncy.data(), nullptr, nullptr, mperm.data(), miperm.data());
  if (status != 1) throw std::runtime_error("symla::computeOrdering: METIS_NodeND failed");
  std::vector<int> perm(n);
  std::vector<char> seen(n, 0);
  for (int k = 0; k < n; ++k) {
    const int64_t v = takeIperm ? miperm[k] : mperm[k];
    if (v < 0 || v >= n || seen[v]) throw std::runtime_error("symla::computeOrdering: METIS returned an invalid permutation");
    seen[v] = 1;
    perm[k] = static_cast<int>(v);
  }
  return perm;
}

}  // namespace symla_host
