// ORACLE -- test infrastructure only (see oracle.hpp).
// The host symbolic analysis (ordering, elimination tree, supernodes;
// symbolic.hpp:195-399 of the reference) compiled into the oracle library
// from the same sources as the GPU path's host side
// (ma57_b200/csrc/host/), so that the CPU baseline can analyse a matrix
// without loading the product library and both sides work on the identical
// permutation and supernode partition.
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../ma57_b200/csrc/host/symbolic.hpp"

namespace {
struct Analysis {
  symla_host::SymbolicFactor sf;
};
void put_error(char* err, int errlen, const char* msg) {
  if (err && errlen > 0) {
    std::strncpy(err, msg, errlen - 1);
    err[errlen - 1] = 0;
  }
}
}  // namespace

extern "C" {

void* oracle_analyze(int n, const int* colptr, const int* rowind, int ordering, int max_relax_size,
                     double max_relax_fill_fraction, char* err, int errlen) {
  try {
    symla_host::SymbolicFactorOptions o;
    o.max_relax_size = max_relax_size;
    o.max_relax_fill_fraction = max_relax_fill_fraction;
    auto* a = new Analysis();
    a->sf = symla_host::analyze(n, colptr, rowind, static_cast<symla_host::OrderingType>(ordering), o);
    return a;
  } catch (const std::exception& e) {
    put_error(err, errlen, e.what());
    return nullptr;
  }
}

void oracle_analysis_sizes(void* h, int* n, int* num_supernodes, long long* pattern_len) {
  const auto& sf = static_cast<Analysis*>(h)->sf;
  *n = sf.etree.n;
  *num_supernodes = static_cast<int>(sf.supernodes.size());
  long long len = 0;
  for (const auto& s : sf.supernodes) len += static_cast<long long>(s.rowPattern.size());
  *pattern_len = len;
}

void oracle_analysis_get(void* h, int* perm, int* parent, int* first, int* ncols, int* ptr, int* rows) {
  const auto& sf = static_cast<Analysis*>(h)->sf;
  std::copy(sf.perm.begin(), sf.perm.end(), perm);
  std::copy(sf.etree.parent.begin(), sf.etree.parent.end(), parent);
  long long off = 0;
  for (size_t i = 0; i < sf.supernodes.size(); ++i) {
    first[i] = sf.supernodes[i].firstCol;
    ncols[i] = sf.supernodes[i].ncols;
    ptr[i] = static_cast<int>(off);
    std::copy(sf.supernodes[i].rowPattern.begin(), sf.supernodes[i].rowPattern.end(), rows + off);
    off += static_cast<long long>(sf.supernodes[i].rowPattern.size());
  }
  ptr[sf.supernodes.size()] = static_cast<int>(off);
}

void oracle_analysis_destroy(void* h) { delete static_cast<Analysis*>(h); }

}  // extern "C"
