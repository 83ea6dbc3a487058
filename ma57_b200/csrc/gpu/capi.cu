// C ABI implementation (include/symla_gpu.h): symbolic entry points, the
// device plan, and the factorize / solve / refine drivers.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../../include/symla_gpu.h"
#include "../host/symbolic.hpp"
#include "context.hpp"
#include "factor_kernels.h"

using namespace symla_gpu;

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace

// Error recording for entry points defined in other translation units.
int symla_gpu::record_error(int code, const std::string& msg) { return set_error(code, msg); }

namespace {

struct CudaError : std::runtime_error {
  cudaError_t err;
  CudaError(cudaError_t e, const char* what) : std::runtime_error(what), err(e) {}
};
struct SymlaError : std::runtime_error {
  int code;
  SymlaError(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define CK(call)                                                                                         \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) {                                                                             \
      char buf_[512];                                                                                    \
      snprintf(buf_, sizeof buf_, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      throw CudaError(e_, buf_);                                                                         \
    }                                                                                                    \
  } while (0)

template <typename F>
int guarded(F&& body) {
  try {
    body();
    return SYMLA_OK;
  } catch (const SymlaError& e) {
    return set_error(e.code, e.what());
  } catch (const CudaError& e) {
    if (e.err == cudaErrorMemoryAllocation) return set_error(SYMLA_ERR_OOM, e.what());
    if (e.err == cudaErrorNoDevice || e.err == cudaErrorInsufficientDriver) return set_error(SYMLA_ERR_NO_DEVICE, e.what());
    return set_error(SYMLA_ERR_CUDA, e.what());
  } catch (const std::bad_alloc&) {
    return set_error(SYMLA_ERR_OOM, "host allocation failed");
  } catch (const std::invalid_argument& e) {
    return set_error(SYMLA_ERR_INVALID, e.what());
  } catch (const std::exception& e) {
    return set_error(SYMLA_ERR_INTERNAL, e.what());
  }
}

// Device bytes a context's creation may still allocate (symla_gpu_set_memory_limit),
// or < 0 for no limit; set for the duration of one symla_gpu_create.
std::atomic<long long> g_create_limit{0};
thread_local long long tl_alloc_budget = -1;

template <typename T>
T* dalloc(size_t count) {
  if (count == 0) count = 1;
  const long long bytes = static_cast<long long>(count * sizeof(T));
  if (tl_alloc_budget >= 0) {
    if (bytes > tl_alloc_budget)
      throw SymlaError(SYMLA_ERR_OOM, "symla_gpu_create: the context's device memory limit is too small for its plan");
    tl_alloc_budget -= bytes;
  }
  void* p = nullptr;
  CK(cudaMalloc(&p, count * sizeof(T)));
  return static_cast<T*>(p);
}

template <typename T>
T* dupload(const std::vector<T>& v, cudaStream_t s) {
  T* p = dalloc<T>(v.size());
  if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return p;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

}  // namespace

extern "C" const char* symla_last_error(void) { return g_last_error.c_str(); }

// ---------------------------------------------------------------------------
// Symbolic
extern "C" int symla_analyze(int n, const int* colptr, const int* rowind, int ordering, int max_relax_size,
                             double max_relax_fill_fraction, symla_symbolic** out) {
  if (!out) return set_error(SYMLA_ERR_INVALID, "symla_analyze: out is NULL");
  *out = nullptr;
  if (n < 0 || (n > 0 && (!colptr || !rowind))) return set_error(SYMLA_ERR_BAD_SIZE, "symla_analyze: bad matrix");
  if (ordering < 0 || ordering > 3) return set_error(SYMLA_ERR_INVALID, "symla::computeOrdering: unknown OrderingType");
  return guarded([&] {
    symla_host::SymbolicFactorOptions opt;
    opt.max_relax_size = max_relax_size;
    opt.max_relax_fill_fraction = max_relax_fill_fraction;
    auto* s = new symla_symbolic();
    try {
      s->sf = symla_host::analyze(n, colptr, rowind, static_cast<symla_host::OrderingType>(ordering), opt);
    } catch (const std::runtime_error& e) {
      delete s;
      throw SymlaError(SYMLA_ERR_INTERNAL, e.what());
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}

extern "C" int symla_compute_ordering(int n, const int* colptr, const int* rowind, int ordering, int* perm) {
  if (n < 0 || (n > 0 && (!colptr || !rowind || !perm)))
    return set_error(SYMLA_ERR_BAD_SIZE, "symla_compute_ordering: bad matrix");
  if (ordering < 0 || ordering > 3) return set_error(SYMLA_ERR_INVALID, "symla::computeOrdering: unknown OrderingType");
  return guarded([&] {
    std::vector<int> p;
    try {
      const auto sym = symla_host::symmetricPatternNoDiag(n, colptr, rowind);
      p = symla_host::computeOrdering(sym, static_cast<symla_host::OrderingType>(ordering));
    } catch (const std::runtime_error& e) {
      throw SymlaError(SYMLA_ERR_INTERNAL, e.what());
    }
    std::copy(p.begin(), p.end(), perm);
  });
}

extern "C" void symla_symbolic_destroy(symla_symbolic* sym) { delete sym; }

extern "C" int symla_symbolic_get_info(const symla_symbolic* sym, symla_symbolic_info* info) {
  if (!sym || !info) return set_error(SYMLA_ERR_INVALID, "null argument");
  const auto& sf = sym->sf;
  info->n = sf.etree.n;
  info->num_supernodes = static_cast<int>(sf.supernodes.size());
  info->num_fundamental = static_cast<int>(sf.fundamentalSupernodes.size());
  info->pattern_len = 0;
  info->storage_nnz = 0;
  for (const auto& s : sf.supernodes) {
    info->pattern_len += static_cast<int64_t>(s.rowPattern.size());
    info->storage_nnz += s.storageNnz();
  }
  info->fundamental_len = 0;
  for (const auto& s : sf.fundamentalSupernodes) info->fundamental_len += static_cast<int64_t>(s.rowPattern.size());
  return SYMLA_OK;
}

namespace {
void export_sn(const std::vector<symla_host::Supernode>& v, int* first, int* ncols, int* ptr, int* rows) {
  int64_t off = 0;
  for (size_t i = 0; i < v.size(); ++i) {
    if (first) first[i] = v[i].firstCol;
    if (ncols) ncols[i] = v[i].ncols;
    if (ptr) ptr[i] = static_cast<int>(off);
    if (rows) std::copy(v[i].rowPattern.begin(), v[i].rowPattern.end(), rows + off);
    off += static_cast<int64_t>(v[i].rowPattern.size());
  }
  if (ptr) ptr[v.size()] = static_cast<int>(off);
}
}  // namespace

extern "C" int symla_symbolic_get(const symla_symbolic* sym, int* perm, int* etree_parent, int* etree_colcount,
                                  int* sn_first, int* sn_ncols, int* sn_ptr, int* sn_rows) {
  if (!sym) return set_error(SYMLA_ERR_INVALID, "null symbolic");
  const auto& sf = sym->sf;
  if (perm) std::copy(sf.perm.begin(), sf.perm.end(), perm);
  if (etree_parent) std::copy(sf.etree.parent.begin(), sf.etree.parent.end(), etree_parent);
  if (etree_colcount) std::copy(sf.etree.colCount.begin(), sf.etree.colCount.end(), etree_colcount);
  export_sn(sf.supernodes, sn_first, sn_ncols, sn_ptr, sn_rows);
  return SYMLA_OK;
}

extern "C" int symla_symbolic_get_fundamental(const symla_symbolic* sym, int* sn_first, int* sn_ncols, int* sn_ptr,
                                              int* sn_rows) {
  if (!sym) return set_error(SYMLA_ERR_INVALID, "null symbolic");
  export_sn(sym->sf.fundamentalSupernodes, sn_first, sn_ncols, sn_ptr, sn_rows);
  return SYMLA_OK;
}

extern "C" int symla_symbolic_import(int n, const int* perm, const int* etree_parent, int num_supernodes,
                                     const int* sn_first, const int* sn_ncols, const int* sn_ptr, const int* sn_rows,
                                     symla_symbolic** out) {
  if (!out || n < 0 || num_supernodes < 0) return set_error(SYMLA_ERR_INVALID, "symla_symbolic_import: bad arguments");
  return guarded([&] {
    auto* s = new symla_symbolic();
    s->sf.perm.assign(perm, perm + n);
    s->sf.etree.n = n;
    s->sf.etree.parent.assign(etree_parent, etree_parent + n);
    s->sf.etree.colCount.assign(n, 0);
    s->sf.supernodes.resize(num_supernodes);
    for (int i = 0; i < num_supernodes; ++i) {
      s->sf.supernodes[i].firstCol = sn_first[i];
      s->sf.supernodes[i].ncols = sn_ncols[i];
      s->sf.supernodes[i].rowPattern.assign(sn_rows + sn_ptr[i], sn_rows + sn_ptr[i + 1]);
    }
    *out = s;
  });
}

// ---------------------------------------------------------------------------
// Plan construction
namespace {

// Leading dimension of a front: m rounded up to even, so that every column
// of a front starts on a 16-byte boundary (bulk copies of whole columns).
int pad_ld(int m) { return m + (m & 1); }

// Builds invmap (length m_parent) and relmap (length cb) for child c of a
// parent whose local row order is given by parentLocal (global -> local).
void build_maps(const std::vector<int>& cbRows, const std::unordered_map<int, int>* g2l,
                const std::vector<int>* parentRows, int mParent, std::vector<int>& invmap, std::vector<int>& relmap) {
  invmap.assign(mParent, -1);
  relmap.resize(cbRows.size());
  for (size_t t = 0; t < cbRows.size(); ++t) {
    int loc;
    if (g2l) {
      auto it = g2l->find(cbRows[t]);
      if (it == g2l->end()) throw SymlaError(SYMLA_ERR_INTERNAL, "extend-add map: child row missing in parent front");
      loc = it->second;
    } else {
      auto it = std::lower_bound(parentRows->begin(), parentRows->end(), cbRows[t]);
      if (it == parentRows->end() || *it != cbRows[t])
        throw SymlaError(SYMLA_ERR_INTERNAL, "extend-add map: child row missing in parent pattern");
      loc = static_cast<int>(it - parentRows->begin());
    }
    relmap[t] = loc;
    invmap[loc] = static_cast<int>(t);
  }
}

void build_level_lists(symla_gpu_ctx* c, const std::vector<int>& frontsOfLevel, LevelLists& L) {
  L.small.clear();
  L.large.clear();
  L.tasks.clear();
  L.all = frontsOfLevel;
  L.small_max_m = L.large_max_m = 0;
  L.panels = 0;
  L.small_flops = 0.0;
  L.assemble_bytes = 0.0;
  L.trailing_flops.clear();
  L.solve_bytes_per_rhs = 0.0;
  L.solve_bytes_fixed = 0.0;
  int tiles = 0;
  for (int s : frontsOfLevel) {
    const auto& f = c->fronts[s];
    // algorithmic factorization flops of the front's nelig 1x1 pivots
    // (lower-triangle convention: r + r(r+1) for trailing size r)
    double ff = 0.0;
    for (int k = 0; k < f.nelig; ++k) {
      const double r = f.m - k - 1;
      ff += r + r * (r + 1);
    }
    const double np = f.nelig;
    L.solve_bytes_fixed += 8.0 * (f.m * np - np * (np - 1) / 2.0) + 4.0 * f.m;
    L.solve_bytes_per_rhs += 8.0 * 2.0 * f.m;
    if (f.m <= kSmallFrontMax) {
      L.small.push_back(s);
      L.small_max_m = std::max(L.small_max_m, f.m);
      L.small_flops += ff;
    } else {
      L.large.push_back(s);
      L.large_max_m = std::max(L.large_max_m, f.m);
      const int panels = (f.nelig + kPanelWidth - 1) / kPanelWidth;
      L.panels = std::max(L.panels, panels);
      if (static_cast<int>(L.trailing_flops.size()) < panels) L.trailing_flops.resize(panels, 0.0);
      for (int it = 0; it < panels; ++it) {
        const int ps = it * kPanelWidth;
        const int p = std::min(kPanelWidth, f.nelig - ps);
        const double mt = f.m - (ps + p);
        L.trailing_flops[it] += static_cast<double>(p) * mt * (mt + 1.0);
      }
      for (int j0 = 0; j0 < f.m; j0 += 32) {
        L.tasks.push_back(s);
        L.tasks.push_back(j0);
        L.tasks.push_back(j0);
        L.tasks.push_back(-1);
      }
      double cbsum = 0.0;
      for (int ch : f.children) {
        const double cb = c->fronts[ch].m - c->fronts[ch].nelig;
        cbsum += cb * (cb + 1) / 2.0;
      }
      L.assemble_bytes += 8.0 * (cbsum + static_cast<double>(f.m) * (f.m + 1) / 2.0);
      const int mt = std::max(0, f.m - std::min(f.nelig, kPanelWidth));
      const int nt = (mt + 127) / 128;
      tiles = std::max(tiles, nt * (nt + 1) / 2);
    }
  }
  if (!L.large.empty() && L.tasks.size() / 4 < 4 * 148) {
    // too few (front, 32 columns) assembly tasks to fill the GPU: split
    // their rows into chunks
    std::vector<int> split;
    for (size_t t = 0; t < L.tasks.size(); t += 4) {
      const int s = L.tasks[t], j0 = L.tasks[t + 1], m = c->fronts[s].m;
      for (int i0 = j0; i0 < m; i0 += kAsmRows) {
        split.push_back(s);
        split.push_back(j0);
        split.push_back(i0);
        split.push_back(i0 + kAsmRows >= m ? -1 : i0 + kAsmRows);
      }
    }
    L.tasks.swap(split);
  }
  if (!L.large.empty()) {
    // one grid over the tiles of every front of the level, in 128 x 128
    // tiles up to one per SM (the update launchers double it: 128 x 64 tiles,
    // two CTAs per SM)
    L.trailing_grid = std::max(1, std::min(tiles * static_cast<int>(L.large.size()), 148));
    // fronts too tall for a full-width cluster panel take narrower panels
    L.panel_width = panel_width_for(L.large_max_m, static_cast<int>(L.large.size()));
    if (L.panel_width != kPanelWidth) {
      L.panels = 0;
      for (int s : L.large) L.panels = std::max(L.panels, (c->fronts[s].nelig + L.panel_width - 1) / L.panel_width);
    }
  } else {
    L.trailing_grid = 0;
  }
}

void free_level_device(LevelLists& L) {
  dfree(L.d_panel_cols);
  L.d_panel_cols = nullptr;
  dfree(L.d_small);
  dfree(L.d_large);
  dfree(L.d_tasks);
  dfree(L.d_all);
  dfree(L.d_fwd_tasks);
  dfree(L.d_bwd_tasks);
  dfree(L.d_tcmaps);
  dfree(L.d_tcws);
  L.d_small = L.d_large = L.d_tasks = L.d_all = nullptr;
  L.d_fwd_tasks = L.d_bwd_tasks = nullptr;
  L.d_tcmaps = nullptr;
  L.d_tcws = nullptr;
  L.tc_grid = 0;
}

// ---------------------------------------------------------------------------
// Mixed-precision far update plumbing: a TF32 hi/lo workspace of
// m x 4 x kTcKpad floats per large front and a TMA tensor map over it
// (32-float x 128-row boxes, 128-byte swizzle, zero fill past row m).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p)
      throw SymlaError(SYMLA_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

size_t tc_level_floats(const symla_gpu_ctx* c, const LevelLists& L) {
  size_t t = 0;
  for (int s : L.large) t += static_cast<size_t>(c->hdesc[s].m) * 4 * kTcKpad;
  return t;
}

void prepare_tc_level(symla_gpu_ctx* c, LevelLists& L, float* base) {
  dfree(L.d_tcmaps);
  dfree(L.d_tcws);
  L.d_tcmaps = nullptr;
  L.d_tcws = nullptr;
  const int nl = static_cast<int>(L.large.size());
  if (nl == 0) return;
  std::vector<CUtensorMap> maps(nl);
  std::vector<float*> ptrs(nl);
  size_t off = 0;
  long long tiles = 0;
  for (int i = 0; i < nl; ++i) {
    const int m = c->hdesc[L.large[i]].m;
    ptrs[i] = base + off;
    off += static_cast<size_t>(m) * 4 * kTcKpad;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(4 * kTcKpad), static_cast<cuuint64_t>(m)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(4 * kTcKpad * sizeof(float))};
    const cuuint32_t box[2] = {32, 128};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_tiled()(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, ptrs[i], dims, strides, box, estr,
                                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw SymlaError(SYMLA_ERR_CUDA, "cuTensorMapEncodeTiled failed for a front workspace");
    const long long nt = (m + 127) / 128;
    tiles += nt * (nt + 1) / 2;
  }
  L.d_tcmaps = dupload(maps, c->stream);
  L.d_tcws = dupload(ptrs, c->stream);
  L.tc_grid = static_cast<int>(std::min<long long>(tiles, 148));
}

// Growth-guard maxima: 2 doubles per large front of the largest level.
void ensure_tc_guard(symla_gpu_ctx* c, const std::vector<LevelLists>& levels) {
  size_t nl = 0;
  for (const auto& L : levels) nl = std::max(nl, L.large.size());
  if (nl <= c->tc_guard_cap) return;
  dfree(c->d_tc_guard);
  c->d_tc_guard = dalloc<double>(2 * nl);
  c->tc_guard_cap = nl;
}

// Static levels: one workspace sized for the largest level, shared by all.
void ensure_tc_static(symla_gpu_ctx* c) {
  if (c->tc_static_ready) return;
  size_t need = 0;
  for (const auto& L : c->levels) need = std::max(need, tc_level_floats(c, L));
  dfree(c->d_tcws);
  c->d_tcws = dalloc<float>(need);
  for (auto& L : c->levels) prepare_tc_level(c, L, c->d_tcws);
  if (!c->d_tc_err) c->d_tc_err = dalloc<int>(1);
  ensure_tc_guard(c, c->levels);
  c->tc_static_ready = true;
}

void upload_level_lists(LevelLists& L, cudaStream_t s) {
  free_level_device(L);
  L.d_small = dupload(L.small, s);
  L.d_large = dupload(L.large, s);
  if (!L.large.empty() && !panel_fits_shared(L.large_max_m))
    L.d_panel_cols = dalloc<double>(2 * static_cast<size_t>(L.large_max_m) * L.large.size());
  L.d_tasks = dupload(L.tasks, s);
  L.d_all = dupload(L.all, s);
}

void build_plan(symla_gpu_ctx* c, const symla_host::SymbolicFactor& sf, const int* colptr, const int* rowind) {
  const int n = c->n;
  const auto& sns = sf.supernodes;
  const int numSN = static_cast<int>(sns.size());
  c->numSN = numSN;
  c->perm = sf.perm;
  c->newIndexOf.assign(n, 0);
  for (int k = 0; k < n; ++k) c->newIndexOf[sf.perm[k]] = k;
  c->rowPatterns.resize(numSN);
  for (int s = 0; s < numSN; ++s) c->rowPatterns[s] = sns[s].rowPattern;

  // supernode tree (multifrontal.hpp:312-332): children in increasing index
  std::vector<int> colToSN(n, -1);
  for (int s = 0; s < numSN; ++s)
    for (int j = sns[s].firstCol; j < sns[s].firstCol + sns[s].ncols; ++j) colToSN[j] = s;
  c->fronts.assign(numSN, HostFront());
  for (int s = 0; s < numSN; ++s) {
    auto& f = c->fronts[s];
    f.firstCol = sns[s].firstCol;
    f.ncols = sns[s].ncols;
    f.nelig = f.ncols;
    f.nextra = 0;
    f.m = static_cast<int>(sns[s].rowPattern.size());
    f.ld = pad_ld(f.m);
    f.rowPattern = &c->rowPatterns[s];
    const int last = f.firstCol + f.ncols - 1;
    const int p = sf.etree.parent[last];
    f.parent = (p == -1) ? -1 : colToSN[p];
  }
  for (int s = 0; s < numSN; ++s)
    if (c->fronts[s].parent >= 0) c->fronts[c->fronts[s].parent].children.push_back(s);
  int numLevels = 0;
  for (int s = 0; s < numSN; ++s) {
    auto& f = c->fronts[s];
    int lv = 0;
    for (int ch : f.children) lv = std::max(lv, c->fronts[ch].level + 1);
    f.level = lv;
    numLevels = std::max(numLevels, lv + 1);
  }
  c->numLevels = numLevels;

  // arena and pools
  std::vector<long long> foff(numSN);
  long long arena = 0, fidxTot = 0, dTot = 0;
  c->fidx_off.assign(numSN, 0);
  c->dpos.assign(numSN, 0);
  c->plan_sum_m2 = 0.0;
  c->plan_max_m = 0;
  for (int s = 0; s < numSN; ++s) {
    const auto& f = c->fronts[s];
    foff[s] = arena;
    arena += static_cast<long long>(f.ld) * f.m;
    c->fidx_off[s] = fidxTot;
    fidxTot += f.m;
    c->dpos[s] = dTot;
    dTot += f.ncols;
    c->plan_sum_m2 += static_cast<double>(f.m) * f.m;
    c->plan_max_m = std::max(c->plan_max_m, f.m);
  }
  c->arena_doubles = static_cast<size_t>(arena);
  c->d_arena = dalloc<double>(arena);
  c->fidx_static.assign(fidxTot, 0);
  for (int s = 0; s < numSN; ++s)
    std::copy(c->rowPatterns[s].begin(), c->rowPatterns[s].end(), c->fidx_static.begin() + c->fidx_off[s]);
  c->d_fidx = dupload(c->fidx_static, c->stream);
  c->d_lperm = dalloc<int>(fidxTot);
  c->d_lpos = dalloc<int>(fidxTot);
  c->d_Dd = dalloc<double>(dTot);
  c->d_Do = dalloc<double>(dTot);
  c->d_pk = dalloc<int8_t>(dTot);

  // extend-add maps
  std::vector<int> mapPool;
  std::vector<std::pair<long long, long long>> linkOffsets;  // (invmap off, relmap off)
  c->hlinks.clear();
  c->link_begin_static.assign(numSN, 0);
  c->link_end_static.assign(numSN, 0);
  std::vector<int> inv, rel, cbRows;
  struct LinkTmp {
    int child;
    long long inv, rel;
    int cb;
  };
  std::vector<LinkTmp> ltmp;
  for (int s = 0; s < numSN; ++s) {
    const auto& f = c->fronts[s];
    c->link_begin_static[s] = static_cast<int>(ltmp.size());
    for (int ch : f.children) {
      const auto& cf = c->fronts[ch];
      cbRows.assign(c->rowPatterns[ch].begin() + cf.ncols, c->rowPatterns[ch].end());
      build_maps(cbRows, nullptr, &c->rowPatterns[s], f.m, inv, rel);
      LinkTmp lt{ch, static_cast<long long>(mapPool.size()), 0, static_cast<int>(cbRows.size())};
      mapPool.insert(mapPool.end(), inv.begin(), inv.end());
      lt.rel = static_cast<long long>(mapPool.size());
      mapPool.insert(mapPool.end(), rel.begin(), rel.end());
      ltmp.push_back(lt);
    }
    c->link_end_static[s] = static_cast<int>(ltmp.size());
  }
  c->d_maps = dupload(mapPool, c->stream);
  c->hlinks.resize(ltmp.size());
  for (size_t i = 0; i < ltmp.size(); ++i) {
    c->hlinks[i].child = ltmp[i].child;
    c->hlinks[i].invmap = c->d_maps + ltmp[i].inv;
    c->hlinks[i].relmap = c->d_maps + ltmp[i].rel;
    c->hlinks[i].cb = ltmp[i].cb;
  }
  c->hlinks_static = c->hlinks;
  c->links_capacity = std::max<size_t>(64, c->hlinks.size() * 2 + 64);
  c->d_links = dalloc<ChildLink>(c->links_capacity);
  if (!c->hlinks.empty())
    CK(cudaMemcpyAsync(c->d_links, c->hlinks.data(), c->hlinks.size() * sizeof(ChildLink), cudaMemcpyHostToDevice,
                       c->stream));

  // A entries: (final column lo, pattern position of hi) -> value index
  struct AEnt {
    int col, pos, j, idx;
  };
  std::vector<AEnt> ents;
  ents.reserve(c->nnz);
  for (int cc = 0; cc < n; ++cc) {
    for (int p = colptr[cc]; p < colptr[cc + 1]; ++p) {
      const int r = rowind[p];
      if (r < cc) continue;
      const int nr = c->newIndexOf[r], nc = c->newIndexOf[cc];
      const int lo = std::min(nr, nc), hi = std::max(nr, nc);
      const int s = colToSN[lo];
      const auto& rp = c->rowPatterns[s];
      auto it = std::lower_bound(rp.begin(), rp.end(), hi);
      if (it == rp.end() || *it != hi) throw SymlaError(SYMLA_ERR_INTERNAL, "A entry outside the supernode pattern");
      ents.push_back(AEnt{lo, static_cast<int>(it - rp.begin()), lo - c->fronts[s].firstCol, p});
    }
  }
  std::sort(ents.begin(), ents.end(), [](const AEnt& a, const AEnt& b) {
    if (a.col != b.col) return a.col < b.col;
    return a.pos < b.pos;
  });
  std::vector<int> acolptr(n + 1, 0), aj(ents.size()), apos(ents.size()), aidx(ents.size());
  for (const auto& e : ents) acolptr[e.col + 1]++;
  for (int i = 0; i < n; ++i) acolptr[i + 1] += acolptr[i];
  for (size_t t = 0; t < ents.size(); ++t) {
    aj[t] = ents[t].j;
    apos[t] = ents[t].pos;
    aidx[t] = ents[t].idx;
  }
  c->d_a_colptr = dupload(acolptr, c->stream);
  c->d_a_j = dupload(aj, c->stream);
  c->d_a_pos = dupload(apos, c->stream);
  c->d_a_idx = dupload(aidx, c->stream);

  // descriptors
  c->hdesc.assign(numSN, FrontDesc());
  for (int s = 0; s < numSN; ++s) {
    const auto& f = c->fronts[s];
    FrontDesc& d = c->hdesc[s];
    d.F = c->d_arena + foff[s];
    d.fidx = c->d_fidx + c->fidx_off[s];
    d.lperm = c->d_lperm + c->fidx_off[s];
    d.lpos = c->d_lpos + c->fidx_off[s];
    d.Dd = c->d_Dd + c->dpos[s];
    d.Do = c->d_Do + c->dpos[s];
    d.pk = c->d_pk + c->dpos[s];
    d.W = nullptr;
    d.m = f.m;
    d.ld = f.ld;
    d.ncols = f.ncols;
    d.nelig = f.nelig;
    d.nextra = 0;
    d.parent = f.parent;
    d.ch_begin = c->link_begin_static[s];
    d.ch_end = c->link_end_static[s];
    d.a_begin = f.firstCol;
    d.a_end = f.firstCol + f.ncols;
    d.level = f.level;
    d.wld = f.m;
  }
  c->hdesc_static = c->hdesc;
  c->d_desc = dupload(c->hdesc, c->stream);
  c->d_state = dalloc<FrontState>(numSN);
  c->d_glob = dalloc<FactorGlobals>(1);

  // levels
  std::vector<std::vector<int>> byLevel(numLevels);
  for (int s = 0; s < numSN; ++s) byLevel[c->fronts[s].level].push_back(s);
  c->levels.assign(numLevels, LevelLists());
  c->level_iters.assign(numLevels, 0);
  c->graph_level_iters.clear();
  for (int l = 0; l < numLevels; ++l) {
    build_level_lists(c, byLevel[l], c->levels[l]);
    upload_level_lists(c->levels[l], c->stream);
  }

  // residual: full symmetric CSR gathered from the stored lower triangle,
  // columns sorted per row; and the stored-entry rows for ||A||
  std::vector<std::vector<std::pair<int, int>>> rows(n);
  std::vector<int> scount(n + 1, 0);
  for (int cc = 0; cc < n; ++cc) {
    for (int p = colptr[cc]; p < colptr[cc + 1]; ++p) {
      const int r = rowind[p];
      scount[r + 1]++;
      if (r < cc) continue;
      rows[r].push_back({cc, p});
      if (r != cc) rows[cc].push_back({r, p});
    }
  }
  std::vector<int> rowptr(n + 1, 0), colind, vidx;
  for (int i = 0; i < n; ++i) {
    std::sort(rows[i].begin(), rows[i].end());
    rowptr[i + 1] = rowptr[i] + static_cast<int>(rows[i].size());
    for (auto& pr : rows[i]) {
      colind.push_back(pr.first);
      vidx.push_back(pr.second);
    }
  }
  for (int i = 0; i < n; ++i) scount[i + 1] += scount[i];
  std::vector<int> svidx(c->nnz), fill(scount.begin(), scount.end() - 1);
  for (int cc = 0; cc < n; ++cc)
    for (int p = colptr[cc]; p < colptr[cc + 1]; ++p) svidx[fill[rowind[p]]++] = p;
  c->nnz_full = static_cast<long long>(colind.size());
  c->d_rowptr = dupload(rowptr, c->stream);
  c->d_colind = dupload(colind, c->stream);
  c->d_vidx = dupload(vidx, c->stream);
  c->d_srowptr = dupload(scount, c->stream);
  c->d_svidx = dupload(svidx, c->stream);
  c->d_perm = dupload(c->perm, c->stream);
  c->d_values = dalloc<double>(c->nnz);
  c->d_sign_final = dalloc<int>(n);
  c->d_front_delta = dalloc<double>(numSN);
  c->d_norms = dalloc<double>(8);
  c->hstate.assign(numSN, FrontState());
  for (int i = 0; i < 8; ++i) CK(cudaEventCreate(&c->ev[i]));
  CK(cudaStreamSynchronize(c->stream));
}

void free_dynamic(symla_gpu_ctx* c) {
  for (void* p : c->dyn_allocs) dfree(p);
  c->dyn_allocs.clear();
  c->dyn_front_blocks.clear();
}

// Reset descriptors / links to the static plan (start of every factorize).
void reset_to_static(symla_gpu_ctx* c) {
  bool changed = false;
  for (int s = 0; s < c->numSN; ++s)
    if (c->fronts[s].replanned) {
      auto& f = c->fronts[s];
      f.replanned = false;
      f.nextra = 0;
      f.nelig = f.ncols;
      f.m = static_cast<int>(c->rowPatterns[s].size());
      f.ld = pad_ld(f.m);
      changed = true;
    }
  if (changed || c->hdesc.size() != c->hdesc_static.size()) {
    c->hdesc = c->hdesc_static;
    c->hlinks = c->hlinks_static;
    CK(cudaMemcpyAsync(c->d_desc, c->hdesc.data(), c->hdesc.size() * sizeof(FrontDesc), cudaMemcpyHostToDevice,
                       c->stream));
    if (!c->hlinks.empty())
      CK(cudaMemcpyAsync(c->d_links, c->hlinks.data(), c->hlinks.size() * sizeof(ChildLink), cudaMemcpyHostToDevice,
                         c->stream));
    c->w_dirty = true;
  }
  // row-index pool back to the symbolic order (pivoting permutes it)
  CK(cudaMemcpyAsync(c->d_fidx, c->fidx_static.data(), c->fidx_static.size() * sizeof(int), cudaMemcpyHostToDevice,
                     c->stream));
  free_dynamic(c);
}

template <typename F>
void timed(symla_gpu_ctx* c, int kind, double flops, double bytes, F&& launch);
void collect_pending(symla_gpu_ctx* c);

KernelOpts make_kernel_opts(symla_gpu_ctx* c, const symla_factor_opts* o) {
  KernelOpts k;
  std::memset(&k, 0, sizeof k);  // padding too: graph reuse compares the bytes
  k.mode = o->mode;
  k.precision = o->precision;
  k.zero_tol = o->zero_tolerance;
  k.rel_floor = o->relative_pivot_floor;
  k.static_delta = o->static_delta;
  k.static_rel_floor = o->static_rel_floor;
  k.static_abs_floor = o->static_abs_floor;
  k.sign_final = (o->mode == SYMLA_MODE_STATIC && o->expected_sign) ? c->d_sign_final : nullptr;
  k.front_delta = (o->mode == SYMLA_MODE_STATIC && o->front_delta) ? c->d_front_delta : nullptr;
  k.values = c->d_values;
  k.a_j = c->d_a_j;
  k.a_pos = c->d_a_pos;
  k.a_idx = c->d_a_idx;
  k.nnz = c->nnz;
  k.chk = c->d_check;
  return k;
}

// ---- checked build: table validation and the status word --------------------
const char* check_code_name(int code) {
  switch (code) {
    case kChkFrontShape: return "front descriptor shape";
    case kChkFrontStorage: return "front storage outside its allocation";
    case kChkRowIndex: return "front row index outside [0, n)";
    case kChkChildLink: return "child link";
    case kChkInvMap: return "parent-to-child map entry";
    case kChkRelMap: return "child-to-parent map entry";
    case kChkAEntry: return "A scatter entry";
    case kChkPivots: return "pivot count";
    case kChkGather: return "contribution-block read";
    case kChkPermute: return "solve permutation entry";
    case kChkSolveRow: return "level-solve row index";
    case kChkWorkspace: return "solve workspace slice";
    default: return "unknown check";
  }
}

void check_status_word(symla_gpu_ctx* c, const char* when) {
  if constexpr (!kCheckedBuild) return;
  CheckWord w{};
  CK(cudaMemcpyAsync(&w, c->d_check, sizeof w, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (w.count != 0) {
    c->unusable = true;
    throw SymlaError(SYMLA_ERR_INTERNAL, std::string("bounds check failed ") + when + ": " +
                                             check_code_name(w.code) + " (front or entry " +
                                             std::to_string(w.where) + ", " + std::to_string(w.count) +
                                             " failed checks); the context is no longer usable");
  }
}

// Validate every front's tables (phase as launch_validate_fronts), then, with
// sync, read the status word: a failure marks the context unusable.
void validate_tables(symla_gpu_ctx* c, int phase, const KernelOpts& ko, const char* when) {
  if constexpr (!kCheckedBuild) return;
  cudaStream_t st = c->stream;
  c->h_ranges.clear();
  c->h_ranges.push_back(c->d_arena);
  c->h_ranges.push_back(c->d_arena + c->arena_doubles);
  for (const auto& b : c->dyn_front_blocks) {
    c->h_ranges.push_back(b.first);
    c->h_ranges.push_back(b.first + b.second);
  }
  if (c->h_ranges.size() > c->ranges_cap) {
    dfree(c->d_ranges);
    c->ranges_cap = c->h_ranges.size() * 2;
    c->d_ranges = dalloc<const double*>(c->ranges_cap);
  }
  CK(cudaMemcpyAsync(c->d_ranges, c->h_ranges.data(), c->h_ranges.size() * sizeof(const double*),
                     cudaMemcpyHostToDevice, st));
  long long wtotal = 0;
  for (int s = 0; s < c->numSN; ++s) wtotal += static_cast<long long>(c->hdesc[s].m) * c->w_nrhs;
  launch_validate_fronts(c->d_desc, c->d_links, c->d_state, nullptr, c->numSN, c->numSN, c->n, c->d_a_colptr, ko,
                         c->d_ranges, static_cast<int>(c->h_ranges.size() / 2), c->d_W, c->d_W + wtotal, c->w_nrhs,
                         phase, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  check_status_word(c, when);
}

// Default choice of the single-CTA panel kernel (see launch_panel_iteration).
constexpr int kSinglePanelMaxFronts = 148;
constexpr int kSinglePanelMaxM = 1024;

void launch_panel_iteration(symla_gpu_ctx* c, const LevelLists& L, int level, const KernelOpts& ko, int dynamic,
                            const int* d_large) {
  cudaStream_t st = c->stream;
  c->cur_level = level;
  const int nl = static_cast<int>(L.large.size());
  timed(c, SYMLA_KERNEL_PANEL, 0.0, 0.0, [&] {
    // the single-CTA panel when asked for (cluster size 1) or, by default in
    // threshold (Bunch-Kaufman) mode, for levels of fewer large fronts than
    // SMs none taller than kSinglePanelMaxM rows: there the cluster's
    // barriers on every pivot-by-pivot decision cost more than its spread of
    // rows saves (static pivoting never leaves the speculative path, so it
    // keeps the cluster)
    const bool single = L.cluster_ctas == 1 || (L.cluster_ctas == 0 && ko.mode == SYMLA_MODE_THRESHOLD &&
                                                nl < kSinglePanelMaxFronts && L.large_max_m <= kSinglePanelMaxM);
    if (c->use_cluster_panel && !single && cluster_size_for(L.large_max_m, nl, L.panel_width) > 0) {
      CK(launch_cluster_panel(c->d_desc, c->d_state, d_large, nl, L.large_max_m, L.panel_width, ko, c->d_glob, level,
                              dynamic, st, L.cluster_ctas));
    } else {
      // fronts too tall for shared memory keep their two working columns in
      // a global buffer (allocated with the level's lists)
      CK(launch_panel(c->d_desc, c->d_state, d_large, nl, L.large_max_m, L.panel_width, ko, c->d_glob, level,
                      dynamic, st, panel_fits_shared(L.large_max_m) ? nullptr : L.d_panel_cols));
    }
  });
  if (ko.precision != SYMLA_PREC_MIXED) {
    // FP64: near and far updates in one launch (disjoint column ranges);
    // timed as the far (Schur-complement) kind
    timed(c, SYMLA_KERNEL_TRAILING, 0.0, 0.0, [&] {
      launch_update_both(c->d_desc, c->d_state, d_large, nl, L.trailing_grid, c->d_glob, level, dynamic, st,
                         L.update_rows == 64 ? 64 : 128);
    });
    return;
  }
  timed(c, SYMLA_KERNEL_NEAR, 0.0, 0.0, [&] {
    launch_update(false, c->d_desc, c->d_state, d_large, nl, L.trailing_grid, c->d_glob, level, dynamic, st,
                  nullptr, L.update_rows == 64 ? 64 : 128);
  });
  if (ko.precision == SYMLA_PREC_MIXED) {
    timed(c, SYMLA_KERNEL_TRAILING, 0.0, 0.0, [&] {
      const int bmax = tc_max_fronts();
      CK(cudaMemsetAsync(c->d_tc_guard, 0, 2 * sizeof(double) * nl, st));
      for (int b = 0; b < nl; b += bmax) {
        const int cnt = std::min(bmax, nl - b);
        double* guard = c->d_tc_guard + 2 * b;
        launch_tc_split(c->d_desc, c->d_state, d_large + b, cnt, L.d_tcws + b, guard, L.large_max_m, c->d_glob,
                        level, dynamic, st);
        launch_tc_far(c->d_desc, c->d_state, d_large + b, cnt, L.d_tcmaps + b, guard, L.tc_grid, c->d_glob, level,
                      dynamic, c->d_tc_err, st);
        // blocks the growth guard kept off the tensor cores
        launch_update(true, c->d_desc, c->d_state, d_large + b, cnt, L.trailing_grid, c->d_glob, level, dynamic,
                      st, guard, L.update_rows == 64 ? 64 : 128);
      }
    });
  } else {
    timed(c, SYMLA_KERNEL_TRAILING, 0.0, 0.0, [&] {
      launch_update(true, c->d_desc, c->d_state, d_large, nl, L.trailing_grid, c->d_glob, level, dynamic, st,
                    nullptr, L.update_rows == 64 ? 64 : 128);
    });
  }
}

// The level's kernels with `iters` panel iterations, no host synchronisation
// (the part a graph launch captures).
void launch_level_planned(symla_gpu_ctx* c, const LevelLists& L, int level, const KernelOpts& ko, int dynamic,
                          const int* d_small, const int* d_large, const int* d_tasks, int iters) {
  cudaStream_t st = c->stream;
  c->cur_level = level;
  if (!L.small.empty())
    timed(c, SYMLA_KERNEL_SMALL, L.small_flops, 0.0, [&] {
      launch_factor_small(c->d_desc, c->d_links, c->d_state, d_small, static_cast<int>(L.small.size()),
                          L.small_max_m, c->d_a_colptr, ko, c->d_glob, level, dynamic, st, L.small_threads);
    });
  if (!L.large.empty()) {
    timed(c, SYMLA_KERNEL_ASSEMBLE, 0.0, L.assemble_bytes, [&] {
      launch_assemble(c->d_desc, c->d_links, c->d_state, d_tasks, static_cast<int>(L.tasks.size() / 4),
                      c->d_a_colptr, ko, c->d_glob, level, dynamic, st);
    });
    for (int it = 0; it < iters; ++it) launch_panel_iteration(c, L, level, ko, dynamic, d_large);
  }
}

void complete_level(symla_gpu_ctx* c, const LevelLists& L, int level, const KernelOpts& ko, int dynamic,
                    const int* d_large, int launched);

// Panel iterations to launch for a level before checking it on the host:
// the planned count, or the most an earlier factorization of the same plan
// needed (the same pattern usually pivots alike).
int level_plan_iters(const symla_gpu_ctx* c, const LevelLists& L, int level) {
  const int seen = level < static_cast<int>(c->level_iters.size()) ? c->level_iters[level] : 0;
  return std::max(L.panels, seen);
}

void launch_level(symla_gpu_ctx* c, const LevelLists& L, int level, const KernelOpts& ko, int dynamic,
                  const int* d_small, const int* d_large, const int* d_tasks) {
  const int iters = level_plan_iters(c, L, level);
  FactorGlobals before{};
  if (c->profiling && !L.large.empty()) {
    CK(cudaMemcpyAsync(&before, c->d_glob, sizeof before, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  launch_level_planned(c, L, level, ko, dynamic, d_small, d_large, d_tasks, iters);
  if (!L.large.empty()) complete_level(c, L, level, ko, dynamic, d_large, iters);
  if (c->profiling && !L.large.empty()) {
    FactorGlobals after{};
    CK(cudaMemcpyAsync(&after, c->d_glob, sizeof after, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->level_panels.size() != static_cast<size_t>(c->numLevels) * 4) c->level_panels.assign(c->numLevels * 4, 0);
    long long* lp = &c->level_panels[static_cast<size_t>(level) * 4];
    lp[0] += after.spec_full - before.spec_full;
    lp[1] += after.spec_partial - before.spec_partial;
    lp[2] += after.spec_failed - before.spec_failed;
    lp[3] += after.seq_panels - before.seq_panels;
  }
  CK(cudaGetLastError());
}

// Flushes (a partner beyond the outer block), 2x2 pivots and speculative
// panels that stop at a failing pivot can leave a front unfinished after
// the planned iterations: run more until done.
void complete_level(symla_gpu_ctx* c, const LevelLists& L, int level, const KernelOpts& ko, int dynamic,
                    const int* d_large, int launched) {
  cudaStream_t st = c->stream;
  {
    const int nl = static_cast<int>(L.large.size());
    int guard = 0;
    for (;;) {
      int unfinished = 0;
      CK(cudaMemsetAsync(c->d_counter, 0, sizeof(int), st));
      launch_count_unfinished(c->d_state, d_large, nl, c->d_counter, st);
      CK(cudaMemcpyAsync(&unfinished, c->d_counter, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (unfinished == 0) break;
      FactorGlobals gl;
      CK(cudaMemcpy(&gl, c->d_glob, sizeof gl, cudaMemcpyDeviceToHost));
      if (!dynamic && gl.delay_level < level) break;  // aborted level, re-run by the delay path
      if (++guard > 4 * L.panels + 64) throw SymlaError(SYMLA_ERR_INTERNAL, "large front did not finish");
      for (int it = 0; it < 4; ++it) launch_panel_iteration(c, L, level, ko, dynamic, d_large);
      launched += 4;
    }
  }
  if (level < static_cast<int>(c->level_iters.size()))
    c->level_iters[level] = std::max(c->level_iters[level], std::min(launched, 4 * L.panels + 64));
  CK(cudaGetLastError());
}

// Graph launch of the static pass: every level with its planned panel
// iterations (or the most an earlier factorization needed) plus slack, each
// level marking itself if a front is still unfinished (the later levels then
// return at once). Captured once per set of kernel options and iteration
// counts and replayed; no host synchronisation inside. A level that ran past
// its count raises it, so the next factorization recaptures with room.
int graph_iters(const symla_gpu_ctx* c, const LevelLists& L, int level) {
  const int n = level_plan_iters(c, L, level);
  return n + n / 8 + 2;
}

void run_static_pass_graph(symla_gpu_ctx* c, const KernelOpts& ko) {
  cudaStream_t st = c->stream;
  std::vector<int> iters(c->numLevels);
  for (int l = 0; l < c->numLevels; ++l) iters[l] = graph_iters(c, c->levels[l], l);
  const bool same = c->graph_exec && std::memcmp(&c->graph_ko, &ko, sizeof ko) == 0 && iters == c->graph_level_iters;
  if (!same) {
    if (c->graph_exec) {
      cudaGraphExecDestroy(c->graph_exec);
      c->graph_exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    const long long counted = c->launches;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int l = 0; l < c->numLevels; ++l) {
      const LevelLists& L = c->levels[l];
      launch_level_planned(c, L, l, ko, 0, L.d_small, L.d_large, L.d_tasks, iters[l]);
      if (!L.large.empty())
        launch_mark_unfinished(c->d_state, L.d_large, static_cast<int>(L.large.size()), c->d_glob, l, st);
    }
    const cudaError_t ec = cudaStreamEndCapture(st, &graph);
    if (ec != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      CK(ec);
    }
    // the captured launches run at every replay, not at the capture
    c->launches = counted;
    size_t nodes = 0;
    c->graph_kernels = 0;
    if (cudaGraphGetNodes(graph, nullptr, &nodes) == cudaSuccess && nodes > 0) {
      std::vector<cudaGraphNode_t> list(nodes);
      if (cudaGraphGetNodes(graph, list.data(), &nodes) == cudaSuccess)
        for (size_t i = 0; i < nodes; ++i) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(list[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++c->graph_kernels;
        }
    }
    const cudaError_t ei = cudaGraphInstantiate(&c->graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ei);
    c->graph_ko = ko;
    c->graph_level_iters = iters;
    ++c->graph_captures;
  }
  CK(cudaGraphLaunch(c->graph_exec, st));
  c->launches += c->graph_kernels;
}

// Re-plan front s whose children delayed columns (multifrontal.hpp:453-479)
// and upload its new descriptor and extend-add maps.
void replan_front(symla_gpu_ctx* c, int s) {
  auto& f = c->fronts[s];
  const auto& rp = c->rowPatterns[s];
  // children's contribution-block row indices, in their current order
  std::vector<std::vector<int>> cbRowsOf(f.children.size());
  std::vector<int> extras;
  for (size_t t = 0; t < f.children.size(); ++t) {
    const int ch = f.children[t];
    const auto& cd = c->hdesc[ch];
    const int np = c->hstate[ch].npiv;
    std::vector<int> rowsAll(cd.m);
    CK(cudaMemcpyAsync(rowsAll.data(), cd.fidx, cd.m * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    cbRowsOf[t].assign(rowsAll.begin() + np, rowsAll.end());
    for (int g : cbRowsOf[t])
      if (!std::binary_search(rp.begin(), rp.end(), g)) extras.push_back(g);
  }
  std::sort(extras.begin(), extras.end());
  extras.erase(std::unique(extras.begin(), extras.end()), extras.end());
  const int nExtra = static_cast<int>(extras.size());
  f.nextra = nExtra;
  f.nelig = f.ncols + nExtra;
  f.m = static_cast<int>(rp.size()) + nExtra;
  f.ld = pad_ld(f.m);
  f.replanned = true;
  std::vector<int> frontIdx(f.m);
  for (int j = 0; j < f.ncols; ++j) frontIdx[j] = f.firstCol + j;
  for (int j = 0; j < nExtra; ++j) frontIdx[f.ncols + j] = extras[j];
  for (int j = f.ncols; j < static_cast<int>(rp.size()); ++j) frontIdx[f.nelig + (j - f.ncols)] = rp[j];
  std::unordered_map<int, int> g2l;
  g2l.reserve(f.m * 2);
  for (int t = 0; t < f.m; ++t) g2l[frontIdx[t]] = t;

  FrontDesc d = c->hdesc[s];
  double* F = dalloc<double>(static_cast<size_t>(f.ld) * f.m);
  c->dyn_allocs.push_back(F);
  c->dyn_front_blocks.push_back({F, static_cast<size_t>(f.ld) * f.m});
  int* fidx = dupload(frontIdx, c->stream);
  c->dyn_allocs.push_back(fidx);
  int* lperm = dalloc<int>(f.m);
  int* lpos = dalloc<int>(f.m);
  c->dyn_allocs.push_back(lperm);
  c->dyn_allocs.push_back(lpos);
  double* Dd = dalloc<double>(f.nelig);
  double* Do = dalloc<double>(f.nelig);
  int8_t* pk = dalloc<int8_t>(f.nelig);
  c->dyn_allocs.push_back(Dd);
  c->dyn_allocs.push_back(Do);
  c->dyn_allocs.push_back(pk);
  d.F = F;
  d.fidx = fidx;
  d.lperm = lperm;
  d.lpos = lpos;
  d.Dd = Dd;
  d.Do = Do;
  d.pk = pk;
  d.m = f.m;
  d.ld = f.ld;
  d.nelig = f.nelig;
  d.nextra = nExtra;
  d.wld = f.m;

  // maps for every child
  std::vector<int> pool, inv, rel;
  std::vector<std::pair<size_t, size_t>> offs;
  for (size_t t = 0; t < f.children.size(); ++t) {
    build_maps(cbRowsOf[t], &g2l, nullptr, f.m, inv, rel);
    offs.push_back({pool.size(), pool.size() + inv.size()});
    pool.insert(pool.end(), inv.begin(), inv.end());
    pool.insert(pool.end(), rel.begin(), rel.end());
  }
  int* dmaps = dupload(pool, c->stream);
  c->dyn_allocs.push_back(dmaps);
  const int begin = static_cast<int>(c->hlinks.size());
  for (size_t t = 0; t < f.children.size(); ++t) {
    ChildLink L;
    L.child = f.children[t];
    L.invmap = dmaps + offs[t].first;
    L.relmap = dmaps + offs[t].second;
    L.cb = static_cast<int>(cbRowsOf[t].size());
    c->hlinks.push_back(L);
  }
  d.ch_begin = begin;
  d.ch_end = static_cast<int>(c->hlinks.size());
  if (c->hlinks.size() > c->links_capacity) {
    size_t cap = c->hlinks.size() * 2;
    ChildLink* nl = dalloc<ChildLink>(cap);
    dfree(c->d_links);
    c->d_links = nl;
    c->links_capacity = cap;
    CK(cudaMemcpyAsync(c->d_links, c->hlinks.data(), c->hlinks.size() * sizeof(ChildLink), cudaMemcpyHostToDevice,
                       c->stream));
  } else {
    CK(cudaMemcpyAsync(c->d_links + begin, c->hlinks.data() + begin, f.children.size() * sizeof(ChildLink),
                       cudaMemcpyHostToDevice, c->stream));
  }
  c->hdesc[s] = d;
  CK(cudaMemcpyAsync(c->d_desc + s, &c->hdesc[s], sizeof(FrontDesc), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->w_dirty = true;
}

void read_states(symla_gpu_ctx* c) {
  CK(cudaMemcpyAsync(c->hstate.data(), c->d_state, c->numSN * sizeof(FrontState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

void run_factorization(symla_gpu_ctx* c, const symla_factor_opts* o, symla_factor_info* info) {
  cudaStream_t st = c->stream;
  reset_to_static(c);
  const KernelOpts ko = make_kernel_opts(c, o);
  CK(cudaMemsetAsync(c->d_state, 0, c->numSN * sizeof(FrontState), st));
  validate_tables(c, 0, ko, "before the factorization");
  FactorGlobals g0{INT_MAX, 0, -1, INT_MAX, 0.0, 0.0, 0.0, 0, 0, 0, 0, c->wait_ns, {0, 0, 0, 0}, 0};
  CK(cudaMemcpyAsync(c->d_glob, &g0, sizeof g0, cudaMemcpyHostToDevice, st));
  const bool mixed = o->precision == SYMLA_PREC_MIXED;
  if (mixed) {
    ensure_tc_static(c);
    CK(cudaMemsetAsync(c->d_tc_err, 0, sizeof(int), st));
    launch_absmax(c->d_values, c->nnz, &c->d_glob->amax, st);  // scale of the growth guard
  }
  CK(cudaEventRecord(c->ev[0], st));
  if (c->use_graph && !c->profiling) {
    run_static_pass_graph(c, ko);
    FactorGlobals gg;
    CK(cudaMemcpyAsync(&gg, c->d_glob, sizeof gg, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (gg.unfinished_level != INT_MAX && gg.unfinished_level <= gg.delay_level) {
      // resume on the host: finish that level, then run the later ones
      const int u = gg.unfinished_level;
      const int none = INT_MAX;
      CK(cudaMemcpyAsync(&c->d_glob->unfinished_level, &none, sizeof none, cudaMemcpyHostToDevice, st));
      ++c->graph_resumes;
      complete_level(c, c->levels[u], u, ko, 0, c->levels[u].d_large, c->graph_level_iters[u]);
      for (int l = u + 1; l < c->numLevels; ++l) {
        const LevelLists& L = c->levels[l];
        launch_level(c, L, l, ko, 0, L.d_small, L.d_large, L.d_tasks);
      }
    }
  } else {
    for (int l = 0; l < c->numLevels; ++l) {
      const LevelLists& L = c->levels[l];
      launch_level(c, L, l, ko, 0, L.d_small, L.d_large, L.d_tasks);
    }
  }
  FactorGlobals g;
  CK(cudaMemcpyAsync(&g, c->d_glob, sizeof g, cudaMemcpyDeviceToHost, st));
  read_states(c);
  bool dynamic = false;
  if (g.delay_level != INT_MAX) {
    // Delayed pivots: fronts above the delaying level were skipped; re-plan
    // and run them level by level with the actual contribution blocks.
    dynamic = true;
    for (int l = g.delay_level + 1; l < c->numLevels; ++l) {
      const LevelLists& Ls = c->levels[l];
      for (int s : Ls.all) {
        bool childDelayed = false;
        for (int ch : c->fronts[s].children)
          if (c->hstate[ch].npiv < c->hdesc[ch].nelig) childDelayed = true;
        if (childDelayed) replan_front(c, s);
      }
      LevelLists L;
      build_level_lists(c, Ls.all, L);
      upload_level_lists(L, st);
      if (mixed && !L.large.empty()) {
        float* ws = dalloc<float>(tc_level_floats(c, L));
        c->dyn_allocs.push_back(ws);
        prepare_tc_level(c, L, ws);
        if (L.large.size() > c->tc_guard_cap) {
          dfree(c->d_tc_guard);
          c->d_tc_guard = dalloc<double>(2 * L.large.size());
          c->tc_guard_cap = L.large.size();
        }
      }
      validate_tables(c, 0, ko, "after re-planning delayed pivots");
      launch_level(c, L, l, ko, 1, L.d_small, L.d_large, L.d_tasks);
      read_states(c);
      free_level_device(L);
    }
  }
  CK(cudaEventRecord(c->ev[1], st));
  CK(cudaEventSynchronize(c->ev[1]));
  collect_pending(c);
  validate_tables(c, 1, ko, "after the factorization");
  if (c->profiling) {
    FactorGlobals gf;
    CK(cudaMemcpy(&gf, c->d_glob, sizeof gf, cudaMemcpyDeviceToHost));
    if (o->precision == SYMLA_PREC_MIXED) {
      c->kstat[SYMLA_KERNEL_TRAILING].flops += gf.flops_far;
      c->kstat[SYMLA_KERNEL_NEAR].flops += gf.flops_near;
    } else {  // one launch does both (timed as the far kind)
      c->kstat[SYMLA_KERNEL_TRAILING].flops += gf.flops_far + gf.flops_near;
    }
  }
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
  {
    FactorGlobals gp;
    CK(cudaMemcpy(&gp, c->d_glob, sizeof gp, cudaMemcpyDeviceToHost));
    c->panel_counts[0] = gp.spec_full;
    c->panel_counts[1] = gp.spec_partial;
    c->panel_counts[2] = gp.spec_failed;
    c->panel_counts[3] = gp.seq_panels;
    for (int i = 0; i < 4; ++i) c->seq_dec_counts[i] = gp.seq_dec[i];
    if (gp.error == kPanelErrTimeout)
      throw SymlaError(SYMLA_ERR_TIMEOUT, "panel factorization: a bulk copy of the panel rows did not complete");
    if (gp.error == kUpdateErrTimeout)
      throw SymlaError(SYMLA_ERR_TIMEOUT, "Schur update: a bulk copy of the staging ring did not complete");
  }
  if (mixed) {
    int tcerr = 0;
    CK(cudaMemcpy(&tcerr, c->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (tcerr & kTcErrDrain) {
      c->unusable = true;
      throw SymlaError(SYMLA_ERR_TIMEOUT,
                       "tensor-core Schur update: a pipeline wait timed out and its drain did not finish; "
                       "the context is no longer usable");
    }
    if (tcerr != 0) throw SymlaError(SYMLA_ERR_TIMEOUT, "tensor-core Schur update: a pipeline wait timed out");
  }
  if (!dynamic) read_states(c);

  // reductions (multifrontal.hpp:795-803)
  symla_factor_info r{};
  c->singular = false;
  c->singularCols.clear();
  double maxGrowth = 1.0;
  for (int s = 0; s < c->numSN; ++s) {
    const FrontState& S = c->hstate[s];
    r.n_pos += S.n_pos;
    r.n_neg += S.n_neg;
    r.n_zero += S.n_zero;
    r.num_perturbed += S.num_perturbed;
    r.total_perturbation += S.perturb;
    r.num_delayed += c->fronts[s].nextra;
    if (S.orig_max > 0) maxGrowth = std::max(maxGrowth, S.running_max / S.orig_max);
    if (S.flags & kFlagSingularRoot) {
      c->singular = true;
      const auto& d = c->hdesc[s];
      std::vector<int> rows(d.m);
      CK(cudaMemcpy(rows.data(), d.fidx, d.m * sizeof(int), cudaMemcpyDeviceToHost));
      for (int i = S.npiv; i < d.m; ++i) c->singularCols.push_back(rows[i]);
    }
  }
  std::sort(c->singularCols.begin(), c->singularCols.end());
  r.singular = c->singular ? 1 : 0;
  r.n_singular = static_cast<int>(c->singularCols.size());
  r.used_dynamic_path = dynamic ? 1 : 0;
  r.max_growth = maxGrowth;
  r.factor_ms = ms;
  c->phase_ms[6] = ms;
  c->last_info = r;
  c->last_precision = o->precision;
  if (info) *info = r;
  c->factorized = true;
}

void ensure_vectors(symla_gpu_ctx* c, int nrhs) {
  if (nrhs <= c->vec_nrhs) return;
  dfree(c->d_Bp);
  dfree(c->d_Z);
  dfree(c->d_Xf);
  dfree(c->d_B);
  dfree(c->d_X);
  dfree(c->d_R);
  dfree(c->d_dX);
  dfree(c->d_Xn);
  dfree(c->d_Rn);
  const size_t len = static_cast<size_t>(c->n) * nrhs;
  c->d_Bp = dalloc<double>(len);
  c->d_Z = dalloc<double>(len);
  c->d_Xf = dalloc<double>(len);
  c->d_B = dalloc<double>(len);
  c->d_X = dalloc<double>(len);
  c->d_R = dalloc<double>(len);
  c->d_dX = dalloc<double>(len);
  c->d_Xn = dalloc<double>(len);
  c->d_Rn = dalloc<double>(len);
  c->vec_nrhs = nrhs;
}

void ensure_workspace(symla_gpu_ctx* c, int nrhs) {
  if (!c->w_dirty && nrhs <= c->w_nrhs) return;
  const int cap = std::max(nrhs, c->w_nrhs);
  long long total = 0;
  for (int s = 0; s < c->numSN; ++s) total += static_cast<long long>(c->hdesc[s].m) * cap;
  dfree(c->d_W);
  c->d_W = dalloc<double>(total);
  long long off = 0;
  for (int s = 0; s < c->numSN; ++s) {
    c->hdesc[s].W = c->d_W + off;
    c->hdesc[s].wld = c->hdesc[s].m;
    off += static_cast<long long>(c->hdesc[s].m) * cap;
  }
  CK(cudaMemcpyAsync(c->d_desc, c->hdesc.data(), c->hdesc.size() * sizeof(FrontDesc), cudaMemcpyHostToDevice,
                     c->stream));
  // keep the static copies' W consistent for fronts that were not re-planned
  for (int s = 0; s < c->numSN; ++s)
    if (!c->fronts[s].replanned) c->hdesc_static[s].W = c->hdesc[s].W;
  c->w_nrhs = cap;
  c->w_dirty = false;
}

// (Re)build the pipelined solve task lists when the fronts' sizes or pivot
// counts differ from the ones the lists were built for.
void ensure_solve_tasks(symla_gpu_ctx* c) {
  std::vector<int> np(c->numSN);
  for (int s = 0; s < c->numSN; ++s) np[s] = c->hstate[s].npiv;
  bool same = (np == c->solve_np) && c->d_flags != nullptr && !c->w_dirty;
  if (same) return;
  const int RB = solve_block_rows();
  std::vector<int> fbase(c->numSN);
  int total = 0;
  for (int s = 0; s < c->numSN; ++s) {
    fbase[s] = total;
    total += (c->hdesc[s].m + RB - 1) / RB;
  }
  if (total > c->flag_count || !c->d_flags) {
    dfree(c->d_flags);
    c->d_flags = dalloc<int>(std::max(1, total));
    CK(cudaMemsetAsync(c->d_flags, 0, std::max(1, total) * sizeof(int), c->stream));
    c->flag_count = total;
    c->solve_epoch = 0;
  }
  dfree(c->d_flag_base);
  c->d_flag_base = dupload(fbase, c->stream);
  // Task shapes per level. Forward: one row block per task (the non-pivot
  // row blocks of a front run concurrently). Backward: with many fronts (at
  // least two per resident CTA) a small front is one task, whose blocks run
  // in order in one CTA with no waits on other CTAs; otherwise a task is one
  // block, and a block with many ancestor-row chunks is split into parts
  // (helpers first) so that one CTA does not walk all of them.
  int slots = 0;
  for (auto& L : c->levels) {
    L.fwd_tasks.clear();
    L.bwd_tasks.clear();
    const bool whole = static_cast<int>(L.all.size()) >= 2 * std::min(c->fwd_resident, c->bwd_resident);
    for (int s : L.all) {
      const int m = c->hdesc[s].m;
      const int nbp = (np[s] + RB - 1) / RB;
      for (int rb = 0; rb * RB < m; ++rb) L.fwd_tasks.push_back(make_int4(s, rb, 0, 0));
      if (whole && m <= 8 * RB) {
        if (nbp > 0) L.bwd_tasks.push_back(make_int4(s, -1, 0, 0));
        continue;
      }
      const int nanc = (m - np[s] + RB - 1) / RB;
      const int P = std::max(1, std::min(8, nanc / 4));
      for (int cb = nbp - 1; cb >= 0; --cb) {
        const int h0 = slots;
        for (int p = 1; p < P; ++p) L.bwd_tasks.push_back(make_int4(s, cb, p, (P << 20) | (h0 + p - 1)));
        L.bwd_tasks.push_back(make_int4(s, cb, 0, (P << 20) | h0));
        slots += P - 1;
      }
    }
    dfree(L.d_fwd_tasks);
    dfree(L.d_bwd_tasks);
    L.d_fwd_tasks = dupload(L.fwd_tasks, c->stream);
    L.d_bwd_tasks = dupload(L.bwd_tasks, c->stream);
  }
  if (slots > c->hslot_count || !c->d_hflags) {
    dfree(c->d_hflags);
    dfree(c->d_hscratch);
    c->d_hflags = dalloc<int>(std::max(1, slots));
    CK(cudaMemsetAsync(c->d_hflags, 0, std::max(1, slots) * sizeof(int), c->stream));
    c->d_hscratch = dalloc<double>(static_cast<size_t>(std::max(1, slots)) * RB * solve_rhs_chunk());
    c->hslot_count = std::max(1, slots);
    c->solve_epoch = std::max(c->solve_epoch, 0);
  }
  c->solve_np = np;
  CK(cudaStreamSynchronize(c->stream));
}

// X := A^{-1} B for device B (ldb) into device X (ldx), both in the
// original index space.
void device_solve(symla_gpu_ctx* c, const double* dB, int ldb, int nrhs, double* dX, int ldx) {
  cudaStream_t st = c->stream;
  ensure_vectors(c, nrhs);
  ensure_workspace(c, nrhs);
  ensure_solve_tasks(c);
  if constexpr (kCheckedBuild) {
    KernelOpts ko;
    std::memset(&ko, 0, sizeof ko);
    ko.a_j = c->d_a_j;
    ko.a_pos = c->d_a_pos;
    ko.a_idx = c->d_a_idx;
    ko.nnz = c->nnz;
    ko.chk = c->d_check;
    validate_tables(c, 2, ko, "before the solve");
  }
  const int n = c->n;
  launch_permute_in(n, nrhs, c->d_perm, dB, ldb, c->d_Bp, st, c->d_check);
  CK(cudaEventRecord(c->ev[2], st));
  const int chunk = solve_rhs_chunk();
  for (int c0 = 0; c0 < nrhs; c0 += chunk) {
    const int nc = std::min(chunk, nrhs - c0);
    const int ef = ++c->solve_epoch;
    for (int l = 0; l < c->numLevels; ++l) {
      const auto& L = c->levels[l];
      const int nt = static_cast<int>(L.fwd_tasks.size());
      const int grid = std::min(nt, c->fwd_resident);
      c->cur_level = l;
      timed(c, SYMLA_KERNEL_FORWARD, 0.0, L.solve_bytes_fixed + nc * L.solve_bytes_per_rhs, [&] {
        CK(launch_forward_pipelined(c->d_desc, c->d_links, c->d_state, L.d_fwd_tasks, nt, grid, c->d_flag_base,
                                    c->d_flags, ef, c->d_solve_err, c->wait_ns, nrhs, c0, c->d_Bp, n, st));
      });
    }
    if (c0 == 0) CK(cudaEventRecord(c->ev[3], st));
    const int eb = ++c->solve_epoch;
    for (int l = c->numLevels - 1; l >= 0; --l) {
      const auto& L = c->levels[l];
      const int nt = static_cast<int>(L.bwd_tasks.size());
      const int grid = std::min(nt, c->bwd_resident);
      c->cur_level = l;
      timed(c, SYMLA_KERNEL_BACKWARD, 0.0, L.solve_bytes_fixed + nc * L.solve_bytes_per_rhs, [&] {
        CK(launch_backward_pipelined(c->d_desc, c->d_state, L.d_bwd_tasks, nt, grid, c->d_flag_base, c->d_flags,
                                     c->d_hflags, c->d_hscratch, eb, c->d_solve_err, c->wait_ns, nrhs, c0, c->d_Xf, n, st));
      });
    }
  }
  c->cur_level = -1;
  CK(cudaEventRecord(c->ev[4], st));
  launch_permute_out(n, nrhs, c->d_perm, c->d_Xf, dX, ldx, st, c->d_check);
  CK(cudaGetLastError());
}

void check_solve_error(symla_gpu_ctx* c) {
  int err = 0;
  CK(cudaMemcpyAsync(&err, c->d_solve_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (err == kSolveErrBounds) {
    c->unusable = true;
    const CheckWord w{1, kChkSolveRow, -1};  // the level kernels report through the solve's error word
    CK(cudaMemcpy(c->d_check, &w, sizeof w, cudaMemcpyHostToDevice));
    throw SymlaError(SYMLA_ERR_INTERNAL,
                     "bounds check failed in the level solve: a row index or a child's workspace row out of range; "
                     "the context is no longer usable");
  }
  if (err != 0) {
    CK(cudaMemsetAsync(c->d_solve_err, 0, sizeof(int), c->stream));
    throw SymlaError(SYMLA_ERR_TIMEOUT, "solve: a pipelined block wait timed out");
  }
  check_status_word(c, "in the solve");
}

void check_usable(symla_gpu_ctx* c) {
  if (c->unusable)
    throw SymlaError(SYMLA_ERR_CUDA,
                     "symla_gpu: the context is no longer usable (an earlier call left its device state untrusted: "
                     "a tensor-core tile's drain timed out, or a bounds check failed); destroy it");
}

void check_solvable(symla_gpu_ctx* c) {
  check_usable(c);
  if (!c->factorized)
    throw SymlaError(SYMLA_ERR_NOT_FACTORIZED, "symla::SymLDLT::solve: factorize() must be called before solve()");
  if (c->singular)
    throw SymlaError(SYMLA_ERR_SINGULAR,
                     "symla::SymLDLT::solve: factorization is numerically singular (see isSingular()/"
                     "singularColumns()); refusing to solve");
}

void upload_values(symla_gpu_ctx* c, const double* values, int on_device) {
  if (c->nnz == 0) return;
  if (on_device)
    CK(cudaMemcpyAsync(c->d_values, values, c->nnz * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  else
    CK(cudaMemcpyAsync(c->d_values, values, c->nnz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
}


cudaEvent_t pool_event(symla_gpu_ctx* c) {
  if (!c->evpool.empty()) {
    cudaEvent_t e = c->evpool.back();
    c->evpool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}

// Brackets a launch with events when profiling; always counts the launch.
template <typename F>
void timed(symla_gpu_ctx* c, int kind, double flops, double bytes, F&& launch) {
  c->launches++;
  if (!c->profiling) {
    launch();
    return;
  }
  cudaEvent_t a = pool_event(c), b = pool_event(c);
  CK(cudaEventRecord(a, c->stream));
  launch();
  CK(cudaEventRecord(b, c->stream));
  c->pending.push_back({a, b, kind, c->cur_level, flops, bytes});
}

void collect_pending(symla_gpu_ctx* c) {
  if (c->pending.empty()) return;
  CK(cudaStreamSynchronize(c->stream));
  for (auto& p : c->pending) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, p.a, p.b));
    auto& k = c->kstat[p.kind];
    k.launches++;
    k.ms += ms;
    k.flops += p.flops;
    k.bytes += p.bytes;
    if (p.level >= 0 && p.level < c->numLevels) {
      if (c->level_kstat.size() != static_cast<size_t>(c->numLevels) * SYMLA_KERNEL_KINDS)
        c->level_kstat.assign(static_cast<size_t>(c->numLevels) * SYMLA_KERNEL_KINDS, {});
      auto& kl = c->level_kstat[static_cast<size_t>(p.level) * SYMLA_KERNEL_KINDS + p.kind];
      kl.launches++;
      kl.ms += ms;
      kl.flops += p.flops;
      kl.bytes += p.bytes;
    }
    c->evpool.push_back(p.a);
    c->evpool.push_back(p.b);
  }
  c->pending.clear();
}
}  // namespace

// ---------------------------------------------------------------------------
extern "C" int symla_gpu_create(const symla_symbolic* sym, int n, const int* colptr, const int* rowind, int device,
                                symla_gpu_ctx** out) {
  if (!out) return set_error(SYMLA_ERR_INVALID, "symla_gpu_create: out is NULL");
  *out = nullptr;
  if (!sym) return set_error(SYMLA_ERR_NOT_ANALYZED, "symla::SymLDLT::factorize: analyzePattern must be called first");
  if (n != sym->sf.etree.n) return set_error(SYMLA_ERR_BAD_SIZE, "symla_gpu_create: matrix size differs from the analysis");
  symla_gpu_ctx* c = new symla_gpu_ctx();
  const long long limit = g_create_limit.load();
  tl_alloc_budget = limit > 0 ? limit : -1;
  const int rc = guarded([&] {
    int count = 0;
    CK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw SymlaError(SYMLA_ERR_NO_DEVICE, "symla_gpu_create: no such CUDA device");
    c->device = device;
    CK(cudaSetDevice(device));
    static bool configured[64] = {};
    if (!configured[device]) {
      CK(configure_factor_kernels());
      CK(configure_cluster_panel());
      CK(configure_tc_far());
      configured[device] = true;
    }
    const char* env = getenv("SYMLA_PANEL");
    c->use_cluster_panel = !(env && std::string(env) == "single");
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->n = n;
    c->nnz = n > 0 ? colptr[n] : 0;
    CK(solve_max_resident(device, &c->fwd_resident, &c->bwd_resident));
    c->d_solve_err = dalloc<int>(1);
    c->d_counter = dalloc<int>(1);
    c->d_check = dalloc<CheckWord>(1);
    CK(cudaMemsetAsync(c->d_solve_err, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->d_check, 0, sizeof(CheckWord), c->stream));
    build_plan(c, sym->sf, colptr, rowind);
  });
  tl_alloc_budget = -1;
  if (rc != SYMLA_OK) {
    symla_gpu_destroy(c);
    return rc;
  }
  *out = c;
  return SYMLA_OK;
}

extern "C" void symla_gpu_destroy(symla_gpu_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  free_dynamic(c);
  for (auto& L : c->levels) free_level_device(L);
  void* ptrs[] = {c->d_arena, c->d_fidx, c->d_lperm, c->d_lpos, c->d_Dd, c->d_Do, c->d_pk, c->d_maps, c->d_desc, c->d_links, c->d_state,
                  c->d_glob, c->d_a_colptr, c->d_a_j, c->d_a_pos, c->d_a_idx, c->d_values, c->d_sign_final,
                  c->d_front_delta, c->d_perm, c->d_rowptr, c->d_colind, c->d_vidx, c->d_srowptr, c->d_svidx, c->d_W,
                  c->d_Bp, c->d_Z, c->d_Xf, c->d_B, c->d_X, c->d_R, c->d_dX, c->d_Xn, c->d_Rn, c->d_norms,
                  c->d_scratch_int, c->d_flag_base, c->d_flags, c->d_solve_err, c->d_counter,
                  c->d_tcws, c->d_tc_err, c->d_tc_guard, c->d_hflags, c->d_hscratch,
                  c->d_gmres, c->d_zero, c->d_gpart, c->d_gcoef, c->d_check, c->d_ranges};
  for (void* p : ptrs) dfree(p);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& p : c->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : c->evpool) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" void symla_factor_opts_default(symla_factor_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->mode = SYMLA_MODE_THRESHOLD;
  o->precision = SYMLA_PREC_FP64;
  o->pivot_threshold = 0.01;
  o->zero_tolerance = 1e-300;
  o->relative_pivot_floor = 1e-12;
  o->static_delta = 0.0;
  o->static_rel_floor = 1e-8;
  o->static_abs_floor = 1e-300;
}

extern "C" int symla_gpu_factorize(symla_gpu_ctx* c, const double* values, int values_on_device,
                                   const symla_factor_opts* opts, symla_factor_info* info) {
  if (!c) return set_error(SYMLA_ERR_NOT_ANALYZED, "symla::SymLDLT::factorize: analyzePattern must be called first");
  symla_factor_opts def;
  symla_factor_opts_default(&def);
  if (!opts) opts = &def;
  if (c->nnz > 0 && !values) return set_error(SYMLA_ERR_INVALID, "symla_gpu_factorize: values is NULL");
  return guarded([&] {
    check_usable(c);
    CK(cudaSetDevice(c->device));
    c->factorized = false;
    upload_values(c, values, values_on_device);
    if (opts->mode == SYMLA_MODE_STATIC) {
      if (opts->expected_sign) {
        std::vector<int> sf(c->n);
        for (int t = 0; t < c->n; ++t) sf[t] = opts->expected_sign[c->perm[t]];
        CK(cudaMemcpyAsync(c->d_sign_final, sf.data(), c->n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
      }
      if (opts->front_delta) {
        CK(cudaMemcpyAsync(c->d_front_delta, opts->front_delta, c->numSN * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
      }
    }
    run_factorization(c, opts, info);
  });
}

extern "C" void symla_regularize_opts_default(symla_regularize_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->initial_delta = 0.0;
  o->max_retries = 10;
  o->growth = 10.0;
  o->static_rel_floor = 1e-8;
  o->static_abs_floor = 1e-300;
  o->expected_sign = nullptr;
  o->kkt_n1 = -1;
  o->kkt_n2 = -1;
  o->precision = SYMLA_PREC_FP64;
  o->front_delta = nullptr;
}

extern "C" int symla_gpu_factorize_regularized(symla_gpu_ctx* c, const double* values, int values_on_device,
                                               const symla_regularize_opts* ro, symla_factor_info* info,
                                               symla_regularize_info* rinfo) {
  if (!c) return set_error(SYMLA_ERR_NOT_ANALYZED, "symla::SymLDLT::factorize: analyzePattern must be called first");
  symla_regularize_opts def;
  symla_regularize_opts_default(&def);
  if (!ro) ro = &def;
  const int n = c->n;
  // solver.hpp:299-317: expected signs in the original index space
  std::vector<int> signs(n, 0);
  bool haveExpectation = false;
  if (ro->expected_sign) {
    signs.assign(ro->expected_sign, ro->expected_sign + n);
    haveExpectation = true;
  } else if (ro->kkt_n1 >= 0) {
    if (ro->kkt_n1 + ro->kkt_n2 != n)
      return set_error(SYMLA_ERR_BAD_SIZE,
                       "symla::SymLDLT::factorize: setKKTBlockSizes(n1, n2) sizes do not sum to the matrix size");
    for (int i = 0; i < ro->kkt_n1; ++i) signs[i] = -1;
    for (int i = ro->kkt_n1; i < n; ++i) signs[i] = +1;
    haveExpectation = true;
  }
  int expectedPos = 0, expectedNeg = 0;
  for (int sgn : signs) {
    if (sgn > 0)
      ++expectedPos;
    else if (sgn < 0)
      ++expectedNeg;
  }
  double delta = ro->initial_delta;
  if (delta <= 0.0) {
    // solver.hpp:346-359: sqrt(eps) * max|A|
    double maxAbs = 0.0;
    if (c->nnz > 0) {
      if (values_on_device) {
        std::vector<double> hv(c->nnz);
        cudaMemcpy(hv.data(), values, c->nnz * sizeof(double), cudaMemcpyDeviceToHost);
        for (double v : hv) maxAbs = std::max(maxAbs, std::fabs(v));
      } else {
        for (int i = 0; i < c->nnz; ++i) maxAbs = std::max(maxAbs, std::fabs(values[i]));
      }
    }
    if (maxAbs <= 0.0) maxAbs = 1.0;
    delta = std::sqrt(std::numeric_limits<double>::epsilon()) * maxAbs;
  }
  symla_factor_opts fo;
  symla_factor_opts_default(&fo);
  fo.mode = SYMLA_MODE_STATIC;
  fo.precision = ro->precision;
  fo.static_rel_floor = ro->static_rel_floor;
  fo.static_abs_floor = ro->static_abs_floor;
  fo.expected_sign = signs.data();
  const int maxAttempts = std::max(1, ro->max_retries + 1);
  symla_regularize_info ri{};
  symla_factor_info fi{};
  for (int attempt = 0; attempt < maxAttempts; ++attempt) {
    fo.static_delta = delta;
    fo.front_delta = (attempt == 0) ? ro->front_delta : nullptr;
    const int rc = symla_gpu_factorize(c, values, values_on_device, &fo, &fi);
    if (rc != SYMLA_OK) return rc;
    ri.retries_used = attempt;
    ri.last_delta = delta;
    const bool fullCoverage = (expectedPos + expectedNeg == n);
    const bool ok = !haveExpectation || (fi.n_zero == 0 && !fi.singular &&
                                         (!fullCoverage || (fi.n_pos == expectedPos && fi.n_neg == expectedNeg)));
    if (ri.attempts < 32) {
      ri.attempt_delta[ri.attempts] = delta;
      ri.attempt_ok[ri.attempts] = ok ? 1 : 0;
    }
    ri.attempts++;
    if (ok) {
      if (info) *info = fi;
      if (rinfo) *rinfo = ri;
      return SYMLA_OK;
    }
    if (attempt + 1 >= maxAttempts) {
      c->factorized = false;
      if (info) *info = fi;
      if (rinfo) *rinfo = ri;
      char buf[640];
      snprintf(buf, sizeof buf,
               "symla::SymLDLT::factorize (Mode::StaticRegularized): inertia-controlled regularization retry budget "
               "(%d retries) exhausted without matching the expected inertia. expected (n_pos=%d, n_neg=%d, "
               "n_zero=0), got (n_pos=%d, n_neg=%d, n_zero=%d, singular=%s) at delta=%g. Refusing to report a "
               "wrong-inertia factorization as successful.",
               ro->max_retries, expectedPos, expectedNeg, fi.n_pos, fi.n_neg, fi.n_zero, fi.singular ? "true" : "false",
               delta);
      return set_error(SYMLA_ERR_RETRY_EXHAUSTED, buf);
    }
    if (attempt == 0 && ro->front_delta && c->numSN > 0) {
      // every front had at least its smallest per-front delta and the
      // inertia still failed: no uniform delta below that is worth a pass
      double dmin = ro->front_delta[0];
      for (int s = 1; s < c->numSN; ++s) dmin = std::min(dmin, ro->front_delta[s]);
      delta = std::max(delta, dmin);
    }
    delta *= ro->growth;
  }
  return SYMLA_OK;
}

extern "C" int symla_gpu_solve(symla_gpu_ctx* c, const double* B, int ldb, int nrhs, double* X, int ldx,
                               int on_device) {
  if (!c) return set_error(SYMLA_ERR_NOT_FACTORIZED, "symla::SymLDLT::solve: factorize() must be called before solve()");
  return guarded([&] {
    check_solvable(c);
    if (nrhs < 0 || ldb < c->n || ldx < c->n)
      throw SymlaError(SYMLA_ERR_BAD_SIZE, "symla::SymLDLT::solve: B.rows() must match the factorized matrix size");
    if (nrhs == 0 || c->n == 0) return;
    CK(cudaSetDevice(c->device));
    const int n = c->n;
    ensure_vectors(c, nrhs);
    CK(cudaEventRecord(c->ev[5], c->stream));
    if (on_device) {
      device_solve(c, B, ldb, nrhs, X, ldx);
    } else {
      CK(cudaMemcpy2DAsync(c->d_B, n * sizeof(double), B, static_cast<size_t>(ldb) * sizeof(double),
                           n * sizeof(double), nrhs, cudaMemcpyHostToDevice, c->stream));
      device_solve(c, c->d_B, n, nrhs, c->d_X, n);
      CK(cudaMemcpy2DAsync(X, static_cast<size_t>(ldx) * sizeof(double), c->d_X, n * sizeof(double),
                           n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaEventRecord(c->ev[6], c->stream));
    CK(cudaEventSynchronize(c->ev[6]));
    collect_pending(c);
    check_solve_error(c);
    float a = 0, b = 0, t = 0;
    cudaEventElapsedTime(&a, c->ev[2], c->ev[3]);
    cudaEventElapsedTime(&b, c->ev[3], c->ev[4]);
    cudaEventElapsedTime(&t, c->ev[5], c->ev[6]);
    c->phase_ms[3] = a;
    c->phase_ms[4] = b;
    c->phase_ms[7] = t;
  });
}

extern "C" int symla_gpu_solve_refine(symla_gpu_ctx* c, const double* values, const double* B, int ldb, int nrhs,
                                      double* X, int ldx, int on_device, int max_iterations, double tolerance,
                                      symla_refine_info* info) {
  if (!c) return set_error(SYMLA_ERR_NOT_FACTORIZED, "symla::SymLDLT::solve: factorize() must be called before solve()");
  return guarded([&] {
    check_solvable(c);
    if (nrhs < 0 || ldb < c->n || ldx < c->n)
      throw SymlaError(SYMLA_ERR_BAD_SIZE, "symla::SymLDLT::solve: B.rows() must match the factorized matrix size");
    CK(cudaSetDevice(c->device));
    const int n = c->n;
    symla_refine_info ri{};
    if (nrhs == 0 || n == 0) {
      if (info) *info = ri;
      return;
    }
    cudaStream_t st = c->stream;
    ensure_vectors(c, nrhs);
    const long long len = static_cast<long long>(n) * nrhs;
    // B -> d_B (compact n x nrhs), values -> d_values
    if (on_device)
      launch_copy2d(n, nrhs, B, ldb, c->d_B, n, st);
    else
      CK(cudaMemcpy2DAsync(c->d_B, n * sizeof(double), B, static_cast<size_t>(ldb) * sizeof(double),
                           n * sizeof(double), nrhs, cudaMemcpyHostToDevice, st));
    if (values) upload_values(c, values, on_device);
    // refine.hpp:106-107
    CK(cudaMemsetAsync(c->d_norms, 0, 8 * sizeof(double), st));
    launch_rowsum_max(n, c->d_srowptr, c->d_svidx, c->d_values, c->d_norms + 0, st);
    launch_absmax(c->d_B, len, c->d_norms + 1, st);
    device_solve(c, c->d_B, n, nrhs, c->d_X, n);
    auto residual_of = [&](const double* Xd, double* Rd, double* out2) {
      CK(cudaMemsetAsync(c->d_norms + 2, 0, 2 * sizeof(double), st));
      timed(c, SYMLA_KERNEL_RESIDUAL, 2.0 * c->nnz_full * nrhs, 12.0 * c->nnz_full + 16.0 * n * nrhs, [&] {
        launch_residual(n, nrhs, c->d_rowptr, c->d_colind, c->d_vidx, c->d_values, Xd, n, c->d_B, n, Rd, st);
      });
      launch_absmax(Rd, len, c->d_norms + 2, st);
      launch_absmax(Xd, len, c->d_norms + 3, st);
      double h[4];
      CK(cudaMemcpyAsync(h, c->d_norms, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      out2[0] = h[2];
      out2[1] = h[3];
      const double denom = h[0] * h[3] + h[1];
      return denom > 0.0 ? h[2] / denom : h[2];
    };
    double nr[2];
    double res = residual_of(c->d_X, c->d_R, nr);
    ri.initial_relative_residual = res;
    ri.final_relative_residual = res;
    for (int it = 0; it < max_iterations; ++it) {
      if (res <= tolerance) break;
      device_solve(c, c->d_R, n, nrhs, c->d_dX, n);
      CK(cudaMemcpyAsync(c->d_Xn, c->d_X, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
      launch_axpy(len, c->d_dX, c->d_Xn, st);
      const double resNew = residual_of(c->d_Xn, c->d_Rn, nr);
      if (!(resNew < res)) break;
      std::swap(c->d_X, c->d_Xn);
      std::swap(c->d_R, c->d_Rn);
      res = resNew;
      ri.iterations = it + 1;
      ri.final_relative_residual = res;
    }
    if (on_device)
      launch_copy2d(n, nrhs, c->d_X, n, X, ldx, st);
    else
      CK(cudaMemcpy2DAsync(X, static_cast<size_t>(ldx) * sizeof(double), c->d_X, n * sizeof(double),
                           n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    collect_pending(c);
    check_solve_error(c);
    if (info) *info = ri;
  });
}

// GMRES-IR (no counterpart in the reference, which lists fixed-precision
// refinement as its limitation, refine.hpp:52-57): outer refinement on the
// FP64 residual with iterativeRefine's stopping and acceptance rules
// (refine.hpp:109-141); each correction A d = r is solved by restarted GMRES
// on M^-1 A, M^-1 the device LDL^T solve, all right-hand sides together
// (classical Gram-Schmidt applied twice; Givens rotations on the host).
extern "C" int symla_gpu_solve_gmres_refine(symla_gpu_ctx* c, const double* values, const double* B, int ldb,
                                            int nrhs, double* X, int ldx, int on_device, int max_outer, int restart,
                                            double tolerance, symla_gmres_info* info) {
  if (!c) return set_error(SYMLA_ERR_NOT_FACTORIZED, "symla::SymLDLT::solve: factorize() must be called before solve()");
  return guarded([&] {
    check_solvable(c);
    if (nrhs < 0 || ldb < c->n || ldx < c->n)
      throw SymlaError(SYMLA_ERR_BAD_SIZE, "symla::SymLDLT::solve: B.rows() must match the factorized matrix size");
    if (restart < 1 || restart > 64)
      throw SymlaError(SYMLA_ERR_INVALID, "symla_gpu_solve_gmres_refine: restart must be in [1, 64]");
    CK(cudaSetDevice(c->device));
    const int n = c->n;
    symla_gmres_info gi{};
    if (nrhs == 0 || n == 0) {
      if (info) *info = gi;
      return;
    }
    cudaStream_t st = c->stream;
    ensure_vectors(c, nrhs);
    const long long len = static_cast<long long>(n) * nrhs;
    const size_t need = static_cast<size_t>(restart + 1) * len;
    if (need > c->gmres_cap) {
      dfree(c->d_gmres);
      c->d_gmres = nullptr;
      c->d_gmres = dalloc<double>(need);
      c->gmres_cap = need;
    }
    if (c->zero_len < n) {
      dfree(c->d_zero);
      c->d_zero = nullptr;
      c->d_zero = dalloc<double>(n);
      c->zero_len = n;
    }
    CK(cudaMemsetAsync(c->d_zero, 0, n * sizeof(double), st));
    const int G = multi_dot_blocks(n);
    const size_t pcap = static_cast<size_t>(restart + 1) * nrhs * G;
    if (pcap > c->gpart_cap) {
      dfree(c->d_gpart);
      c->d_gpart = nullptr;
      c->d_gpart = dalloc<double>(pcap);
      c->gpart_cap = pcap;
    }
    const size_t ccap = static_cast<size_t>(restart + 1) * nrhs;
    if (ccap > c->gcoef_cap) {
      dfree(c->d_gcoef);
      c->d_gcoef = nullptr;
      c->d_gcoef = dalloc<double>(ccap);
      c->gcoef_cap = ccap;
    }
    double* V = c->d_gmres;
    const long long vs = len;
    if (on_device)
      launch_copy2d(n, nrhs, B, ldb, c->d_B, n, st);
    else
      CK(cudaMemcpy2DAsync(c->d_B, n * sizeof(double), B, static_cast<size_t>(ldb) * sizeof(double),
                           n * sizeof(double), nrhs, cudaMemcpyHostToDevice, st));
    if (values) upload_values(c, values, on_device);
    CK(cudaMemsetAsync(c->d_norms, 0, 8 * sizeof(double), st));
    launch_rowsum_max(n, c->d_srowptr, c->d_svidx, c->d_values, c->d_norms + 0, st);
    launch_absmax(c->d_B, len, c->d_norms + 1, st);
    device_solve(c, c->d_B, n, nrhs, c->d_X, n);
    auto residual_of = [&](const double* Xd, double* Rd) {
      CK(cudaMemsetAsync(c->d_norms + 2, 0, 2 * sizeof(double), st));
      launch_residual(n, nrhs, c->d_rowptr, c->d_colind, c->d_vidx, c->d_values, Xd, n, c->d_B, n, Rd, st);
      launch_absmax(Rd, len, c->d_norms + 2, st);
      launch_absmax(Xd, len, c->d_norms + 3, st);
      double h[4];
      CK(cudaMemcpyAsync(h, c->d_norms, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      const double denom = h[0] * h[3] + h[1];
      return denom > 0.0 ? h[2] / denom : h[2];
    };
    std::vector<double> part(pcap), coef(ccap);
    // out[i nrhs + cc] = V_i[:, cc] . W[:, cc], partials summed in a fixed order
    auto dots = [&](int nvec, const double* Vb, const double* W, std::vector<double>& out) {
      launch_multi_dot(n, nrhs, nvec, Vb, vs, W, c->d_gpart, st);
      CK(cudaMemcpyAsync(part.data(), c->d_gpart, static_cast<size_t>(nvec) * nrhs * G * sizeof(double),
                         cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      out.assign(static_cast<size_t>(nvec) * nrhs, 0.0);
      for (size_t t = 0; t < out.size(); ++t) {
        double sum = 0.0;
        for (int b = 0; b < G; ++b) sum += part[t * G + b];
        out[t] = sum;
      }
    };
    auto sub = [&](int nvec, const double* Vb, const std::vector<double>& cf, double* W) {
      CK(cudaMemcpyAsync(c->d_gcoef, cf.data(), static_cast<size_t>(nvec) * nrhs * sizeof(double),
                         cudaMemcpyHostToDevice, st));
      launch_multi_axpy(n, nrhs, nvec, Vb, vs, c->d_gcoef, W, st);
    };
    auto scale = [&](const std::vector<double>& alpha, double* W) {
      CK(cudaMemcpyAsync(c->d_gcoef, alpha.data(), nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
      launch_col_scale(n, nrhs, c->d_gcoef, W, W, st);
    };
    double res = residual_of(c->d_X, c->d_R);
    gi.initial_relative_residual = gi.final_relative_residual = res;
    const int ldh = restart + 1;
    std::vector<double> H(static_cast<size_t>(nrhs) * ldh * restart), g(static_cast<size_t>(nrhs) * ldh),
        cs(static_cast<size_t>(nrhs) * restart), sn(static_cast<size_t>(nrhs) * restart), beta(nrhs), nn, d1, hs,
        alpha(nrhs);
    for (int outer = 0; outer < max_outer && res > tolerance; ++outer) {
      // z = M^-1 r into v_0, normalised per column
      device_solve(c, c->d_R, n, nrhs, V, n);
      dots(1, V, V, nn);
      for (int cc = 0; cc < nrhs; ++cc) {
        beta[cc] = std::sqrt(std::max(nn[cc], 0.0));
        alpha[cc] = beta[cc] > 0.0 ? 1.0 / beta[cc] : 0.0;
        std::fill(g.begin() + static_cast<size_t>(cc) * ldh, g.begin() + static_cast<size_t>(cc + 1) * ldh, 0.0);
        g[static_cast<size_t>(cc) * ldh] = beta[cc];
      }
      scale(alpha, V);
      std::vector<char> active(nrhs);
      for (int cc = 0; cc < nrhs; ++cc) active[cc] = beta[cc] > 0.0;
      int kdone = 0;
      for (int k = 0; k < restart; ++k) {
        double* vk1 = V + static_cast<long long>(k + 1) * vs;
        // u = M^-1 (0 - A v_k) = -M^-1 A v_k
        launch_residual(n, nrhs, c->d_rowptr, c->d_colind, c->d_vidx, c->d_values, V + static_cast<long long>(k) * vs,
                        n, c->d_zero, 0, c->d_Rn, st);
        device_solve(c, c->d_Rn, n, nrhs, vk1, n);
        hs.assign(static_cast<size_t>(k + 1) * nrhs, 0.0);
        for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
          dots(k + 1, V, vk1, d1);
          sub(k + 1, V, d1, vk1);
          for (size_t t = 0; t < hs.size(); ++t) hs[t] += d1[t];
        }
        dots(1, vk1, vk1, nn);
        bool all_done = true;
        for (int cc = 0; cc < nrhs; ++cc) {
          double* Hc = H.data() + static_cast<size_t>(cc) * ldh * restart;
          double* gc = g.data() + static_cast<size_t>(cc) * ldh;
          double* csc = cs.data() + static_cast<size_t>(cc) * restart;
          double* snc = sn.data() + static_cast<size_t>(cc) * restart;
          const double hk1 = std::sqrt(std::max(nn[cc], 0.0));
          alpha[cc] = hk1 > 0.0 ? -1.0 / hk1 : 0.0;  // v_{k+1} = w / h = -u / h
          if (!active[cc]) continue;
          for (int i = 0; i <= k; ++i) Hc[i + k * ldh] = -hs[static_cast<size_t>(i) * nrhs + cc];
          Hc[k + 1 + k * ldh] = hk1;
          for (int i = 0; i < k; ++i) {
            const double t = csc[i] * Hc[i + k * ldh] + snc[i] * Hc[i + 1 + k * ldh];
            Hc[i + 1 + k * ldh] = -snc[i] * Hc[i + k * ldh] + csc[i] * Hc[i + 1 + k * ldh];
            Hc[i + k * ldh] = t;
          }
          const double a = Hc[k + k * ldh], b = Hc[k + 1 + k * ldh];
          const double r = std::hypot(a, b);
          csc[k] = r > 0.0 ? a / r : 1.0;
          snc[k] = r > 0.0 ? b / r : 0.0;
          Hc[k + k * ldh] = r;
          Hc[k + 1 + k * ldh] = 0.0;
          gc[k + 1] = -snc[k] * gc[k];
          gc[k] = csc[k] * gc[k];
          // this column's Krylov space is exhausted or its residual estimate
          // is below the inner tolerance
          if (hk1 == 0.0 || std::fabs(gc[k + 1]) <= 1e-13 * beta[cc]) active[cc] = 0;
          all_done = all_done && !active[cc];
        }
        scale(alpha, vk1);
        kdone = k + 1;
        ++gi.inner_iterations;
        if (all_done) break;
      }
      // y = R^-1 g per column (upper triangular, kdone x kdone); x += V y
      for (int cc = 0; cc < nrhs; ++cc) {
        const double* Hc = H.data() + static_cast<size_t>(cc) * ldh * restart;
        const double* gc = g.data() + static_cast<size_t>(cc) * ldh;
        std::vector<double> y(kdone, 0.0);
        if (beta[cc] > 0.0)
          for (int i = kdone - 1; i >= 0; --i) {
            double t = gc[i];
            for (int j = i + 1; j < kdone; ++j) t -= Hc[i + j * ldh] * y[j];
            y[i] = Hc[i + i * ldh] != 0.0 ? t / Hc[i + i * ldh] : 0.0;
          }
        for (int i = 0; i < kdone; ++i) coef[static_cast<size_t>(i) * nrhs + cc] = -y[i];
      }
      CK(cudaMemcpyAsync(c->d_Xn, c->d_X, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
      sub(kdone, V, coef, c->d_Xn);
      const double resNew = residual_of(c->d_Xn, c->d_Rn);
      gi.outer_iterations = outer + 1;
      if (!(resNew < res)) break;  // keep the better iterate (refine.hpp:121-141)
      std::swap(c->d_X, c->d_Xn);
      std::swap(c->d_R, c->d_Rn);
      res = resNew;
      gi.final_relative_residual = res;
    }
    if (on_device)
      launch_copy2d(n, nrhs, c->d_X, n, X, ldx, st);
    else
      CK(cudaMemcpy2DAsync(X, static_cast<size_t>(ldx) * sizeof(double), c->d_X, n * sizeof(double),
                           n * sizeof(double), nrhs, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    collect_pending(c);
    check_solve_error(c);
    if (info) *info = gi;
  });
}

extern "C" int symla_gpu_singular_cols(symla_gpu_ctx* c, int* cols, int cap) {
  if (!c) return 0;
  const int k = static_cast<int>(c->singularCols.size());
  for (int i = 0; i < k && i < cap; ++i) cols[i] = c->singularCols[i];
  return k;
}

extern "C" int symla_gpu_num_fronts(symla_gpu_ctx* c) { return c ? c->numSN : 0; }

extern "C" int symla_gpu_front_size(symla_gpu_ctx* c, int si, int* m, int* npiv) {
  if (!c || si < 0 || si >= c->numSN) return set_error(SYMLA_ERR_INVALID, "front index out of range");
  if (m) *m = c->hdesc[si].m;
  if (npiv) *npiv = c->factorized ? c->hstate[si].npiv : 0;
  return SYMLA_OK;
}

extern "C" int symla_gpu_front_get(symla_gpu_ctx* c, int si, int* row_indices, double* L, double* d_diag,
                                   double* d_off, int* piv_start, int* piv_kind) {
  if (!c || si < 0 || si >= c->numSN) return set_error(SYMLA_ERR_INVALID, "front index out of range");
  int nblocks = 0;
  const int rc = guarded([&] {
    if (!c->factorized) throw SymlaError(SYMLA_ERR_NOT_FACTORIZED, "not factorized");
    const FrontDesc& d = c->hdesc[si];
    const int m = d.m, np = c->hstate[si].npiv;
    if (row_indices) CK(cudaMemcpy(row_indices, d.fidx, m * sizeof(int), cudaMemcpyDeviceToHost));
    if (L && np > 0) {
      std::vector<double> F(static_cast<size_t>(d.ld) * np);
      CK(cudaMemcpy(F.data(), d.F, F.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < m; ++i) L[i + static_cast<size_t>(j) * m] = (i >= j) ? F[i + static_cast<size_t>(j) * d.ld] : 0.0;
    }
    std::vector<int8_t> pk(np);
    if (np > 0) CK(cudaMemcpy(pk.data(), d.pk, np, cudaMemcpyDeviceToHost));
    if (d_diag && np > 0) CK(cudaMemcpy(d_diag, d.Dd, np * sizeof(double), cudaMemcpyDeviceToHost));
    if (d_off && np > 0) CK(cudaMemcpy(d_off, d.Do, np * sizeof(double), cudaMemcpyDeviceToHost));
    for (int k = 0; k < np; ++k) {
      if (pk[k] == 2) continue;
      if (piv_start) piv_start[nblocks] = k;
      if (piv_kind) piv_kind[nblocks] = (pk[k] == 1) ? 1 : 0;
      ++nblocks;
    }
  });
  return rc == SYMLA_OK ? nblocks : -rc;
}

extern "C" void* symla_gpu_stream(symla_gpu_ctx* c) { return c ? c->stream : nullptr; }

extern "C" int symla_gpu_phase_ms(symla_gpu_ctx* c, float* ms, int cap) {
  if (!c) return 0;
  for (int i = 0; i < cap && i < 8; ++i) ms[i] = c->phase_ms[i];
  return 8;
}

extern "C" int symla_gpu_plan_stats(symla_gpu_ctx* c, double* out, int cap) {
  if (!c) return 0;
  double v[15] = {0};
  v[0] = c->numSN;
  v[1] = c->numLevels;
  v[2] = c->plan_max_m;
  v[3] = c->plan_sum_m2;
  if (c->factorized) {
    double flops = 0.0, nnzL = 0.0;
    for (int s = 0; s < c->numSN; ++s) {
      const FrontDesc& d = c->hdesc[s];
      const int np = c->hstate[s].npiv, m = d.m;
      std::vector<int8_t> pk(np);
      if (np > 0) cudaMemcpy(pk.data(), d.pk, np, cudaMemcpyDeviceToHost);
      for (int k = 0; k < np;) {
        if (pk[k] == 1) {
          const double r = m - k - 2;
          flops += 3 * r + 2 * r * (r + 1);
          k += 2;
        } else {
          const double r = m - k - 1;
          flops += r + r * (r + 1);
          k += 1;
        }
      }
      nnzL += static_cast<double>(m) * np - static_cast<double>(np) * (np - 1) / 2.0;
    }
    v[4] = flops;
    v[5] = nnzL;
  }
  v[6] = static_cast<double>(c->arena_doubles);
  for (int i = 0; i < 4; ++i) v[7 + i] = c->panel_counts[i];
  for (int i = 0; i < 4; ++i) v[11 + i] = c->seq_dec_counts[i];
  for (int i = 0; i < cap && i < 15; ++i) out[i] = v[i];
  return 15;
}

extern "C" int symla_gpu_level_info(symla_gpu_ctx* c, int level, int* out6) {
  if (!c || level < 0 || level >= c->numLevels || !out6) return set_error(SYMLA_ERR_INVALID, "bad arguments");
  const auto& L = c->levels[level];
  out6[0] = static_cast<int>(L.small.size());
  out6[1] = L.small_max_m;
  out6[2] = static_cast<int>(L.large.size());
  out6[3] = L.large_max_m;
  out6[4] = L.small_threads;
  out6[5] = L.cluster_ctas;
  return SYMLA_OK;
}

extern "C" int symla_gpu_set_level_schedule(symla_gpu_ctx* c, int level, int small_threads, int cluster_ctas) {
  if (!c || level < 0 || level >= c->numLevels) return set_error(SYMLA_ERR_INVALID, "level out of range");
  if ((small_threads != 0 && small_threads != 32 && small_threads != 128 && small_threads != 256) ||
      (cluster_ctas != 0 && cluster_ctas != 1 && cluster_ctas != 2 && cluster_ctas != 4 && cluster_ctas != 8 &&
       cluster_ctas != 16))
    return set_error(SYMLA_ERR_INVALID,
                     "symla_gpu_set_level_schedule: small_threads in {0,32,128,256}, cluster_ctas in {0,1,2,4,8,16}");
  auto& L = c->levels[level];
  if (L.small_threads == small_threads && L.cluster_ctas == cluster_ctas) return SYMLA_OK;
  return guarded([&] {
    // the single-CTA panel keeps its two working columns in a global buffer
    // when they do not fit its shared memory
    if (cluster_ctas == 1 && !L.large.empty() && !panel_fits_shared(L.large_max_m) && !L.d_panel_cols)
      L.d_panel_cols = dalloc<double>(2 * static_cast<size_t>(L.large_max_m) * L.large.size());
    L.small_threads = small_threads;
    L.cluster_ctas = cluster_ctas;
    if (c->graph_exec) {  // the captured launches used the old shapes
      cudaGraphExecDestroy(c->graph_exec);
      c->graph_exec = nullptr;
    }
  });
}

extern "C" int symla_gpu_set_level_update_rows(symla_gpu_ctx* c, int level, int rows) {
  if (!c || level < 0 || level >= c->numLevels) return set_error(SYMLA_ERR_INVALID, "level out of range");
  if (rows != 0 && rows != 64 && rows != 128)
    return set_error(SYMLA_ERR_INVALID, "symla_gpu_set_level_update_rows: rows in {0, 64, 128}");
  auto& L = c->levels[level];
  if (L.update_rows != rows) {
    L.update_rows = rows;
    if (c->graph_exec) {  // the captured launches used the old shape
      cudaGraphExecDestroy(c->graph_exec);
      c->graph_exec = nullptr;
    }
  }
  return SYMLA_OK;
}

extern "C" int symla_gpu_level_update_rows(symla_gpu_ctx* c, int level, int* rows) {
  if (!c || !rows || level < 0 || level >= c->numLevels) return set_error(SYMLA_ERR_INVALID, "level out of range");
  *rows = c->levels[level].update_rows == 64 ? 64 : 128;
  return SYMLA_OK;
}

extern "C" int symla_gpu_set_memory_limit(long long bytes) {
  if (bytes < 0) return set_error(SYMLA_ERR_INVALID, "symla_gpu_set_memory_limit: negative limit");
  g_create_limit.store(bytes);
  return SYMLA_OK;
}

extern "C" int symla_gpu_set_wait_limit_ns(symla_gpu_ctx* c, unsigned long long ns) {
  if (!c) return set_error(SYMLA_ERR_INVALID, "null context");
  c->wait_ns = ns == 0 ? symla_gpu::kDefaultWaitNs : ns;
  return SYMLA_OK;
}

extern "C" int symla_gpu_set_graph(symla_gpu_ctx* c, int enable) {
  if (!c) return set_error(SYMLA_ERR_INVALID, "null context");
  c->use_graph = enable != 0;
  return SYMLA_OK;
}

extern "C" int symla_gpu_graph_stats(symla_gpu_ctx* c, int* captures, int* resumes) {
  if (!c) return set_error(SYMLA_ERR_INVALID, "null context");
  if (captures) *captures = c->graph_captures;
  if (resumes) *resumes = c->graph_resumes;
  return SYMLA_OK;
}

extern "C" int symla_gpu_set_profiling(symla_gpu_ctx* c, int enable) {
  if (!c) return set_error(SYMLA_ERR_INVALID, "null context");
  c->profiling = enable != 0;
  return SYMLA_OK;
}

extern "C" int symla_gpu_kernel_stats(symla_gpu_ctx* c, int kind, double* out4) {
  if (!c || kind < 0 || kind >= SYMLA_KERNEL_KINDS || !out4) return set_error(SYMLA_ERR_INVALID, "bad arguments");
  const auto& k = c->kstat[kind];
  out4[0] = static_cast<double>(k.launches);
  out4[1] = k.ms;
  out4[2] = k.flops;
  out4[3] = k.bytes;
  return SYMLA_OK;
}

extern "C" int symla_gpu_level_kernel_stats(symla_gpu_ctx* c, int level, int kind, double* out4) {
  if (!c || kind < 0 || kind >= SYMLA_KERNEL_KINDS || !out4 || level < 0 || level >= c->numLevels)
    return set_error(SYMLA_ERR_INVALID, "bad arguments");
  symla_gpu_ctx::KStat k;
  if (c->level_kstat.size() == static_cast<size_t>(c->numLevels) * SYMLA_KERNEL_KINDS)
    k = c->level_kstat[static_cast<size_t>(level) * SYMLA_KERNEL_KINDS + kind];
  out4[0] = static_cast<double>(k.launches);
  out4[1] = k.ms;
  out4[2] = k.flops;
  out4[3] = k.bytes;
  return SYMLA_OK;
}

extern "C" int symla_gpu_level_panel_stats(symla_gpu_ctx* c, int level, long long* out4) {
  if (!c || !out4 || level < 0 || level >= c->numLevels) return set_error(SYMLA_ERR_INVALID, "bad arguments");
  for (int t = 0; t < 4; ++t)
    out4[t] = c->level_panels.size() == static_cast<size_t>(c->numLevels) * 4
                  ? c->level_panels[static_cast<size_t>(level) * 4 + t]
                  : 0;
  return SYMLA_OK;
}

extern "C" void symla_gpu_reset_kernel_stats(symla_gpu_ctx* c) {
  if (!c) return;
  for (auto& k : c->kstat) k = symla_gpu_ctx::KStat();
  c->level_kstat.clear();
  c->level_panels.clear();
  c->launches = 0;
}

extern "C" long long symla_gpu_launch_count(symla_gpu_ctx* c) { return c ? c->launches : 0; }

extern "C" int symla_gpu_checked_build(void) { return kCheckedBuild ? 1 : 0; }

extern "C" int symla_gpu_check_status(symla_gpu_ctx* c, int* count, int* code, long long* where) {
  if (!c || !count || !code || !where) return set_error(SYMLA_ERR_INVALID, "symla_gpu_check_status: NULL argument");
  return guarded([&] {
    CheckWord w{};
    CK(cudaMemcpyAsync(&w, c->d_check, sizeof w, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *count = w.count;
    *code = w.code;
    *where = w.where;
  });
}
