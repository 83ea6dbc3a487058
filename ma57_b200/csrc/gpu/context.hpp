// Device context behind the C ABI (include/symla_gpu.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../host/symbolic.hpp"
#include "common.cuh"

struct symla_symbolic {
  symla_host::SymbolicFactor sf;
};

namespace symla_gpu {

// Host mirror of one front's current layout.
struct HostFront {
  int firstCol = 0, ncols = 0, nelig = 0, nextra = 0;
  int m = 0, ld = 0;
  int parent = -1, level = 0;
  std::vector<int> children;
  const std::vector<int>* rowPattern = nullptr;
  bool replanned = false;
};

struct LevelLists {
  std::vector<int> small;      // fronts with m <= kSmallFrontMax
  int small_max_m = 0;
  std::vector<int> large;      // other fronts
  int large_max_m = 0;
  int small_threads = 0;       // tile schedule (autotuner): small-front kernel width, 0 = by size
  int cluster_ctas = 0;        // panel cluster size, 0 = by size
  int update_rows = 0;         // rows per Schur-update tile (64 or 128), 0 = 128
  int panels = 0;              // panel iterations needed
  int panel_width = 32;        // pivots per panel (narrower for fronts too tall for a full-width cluster panel)
  double* d_panel_cols = nullptr;  // single-CTA panel kernel, fronts too tall for shared memory: 2 m per front
  int trailing_grid = 0;
  std::vector<int> tasks;      // assembly tasks (front, column block) for large fronts
  std::vector<int> all;        // every front of the level (solve)
  // algorithmic work estimates (instrumentation)
  double small_flops = 0.0;
  double assemble_bytes = 0.0;
  std::vector<double> trailing_flops;  // per panel iteration
  double solve_bytes_fixed = 0.0;
  double solve_bytes_per_rhs = 0.0;
  // pipelined solve tasks {front, block}
  std::vector<int4> fwd_tasks, bwd_tasks;
  int4* d_fwd_tasks = nullptr;
  int4* d_bwd_tasks = nullptr;
  // device copies (static plan)
  int* d_small = nullptr;
  int* d_large = nullptr;
  int* d_tasks = nullptr;
  int* d_all = nullptr;
  // mixed-precision far update: per large front (list order) its TF32
  // workspace and the tensor map over it (built on first use)
  CUtensorMap* d_tcmaps = nullptr;
  float** d_tcws = nullptr;
  int tc_grid = 0;
};

struct DeviceBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Sets the message symla_last_error returns; returns code.
int record_error(int code, const std::string& msg);

}  // namespace symla_gpu

struct symla_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n = 0;
  int nnz = 0;
  long long nnz_full = 0;
  int numSN = 0;
  int numLevels = 0;

  std::vector<int> perm;  // final -> original
  std::vector<int> newIndexOf;
  std::vector<symla_gpu::HostFront> fronts;
  std::vector<std::vector<int>> rowPatterns;  // owned copy of supernode patterns
  std::vector<symla_gpu::LevelLists> levels;
  std::vector<symla_gpu::FrontDesc> hdesc;
  std::vector<symla_gpu::FrontDesc> hdesc_static;
  std::vector<symla_gpu::ChildLink> hlinks;
  std::vector<symla_gpu::ChildLink> hlinks_static;
  std::vector<int> link_begin_static, link_end_static;

  // device: static plan
  double* d_arena = nullptr;
  size_t arena_doubles = 0;
  int* d_fidx = nullptr;       // per-front row index pool (static layout)
  int* d_lperm = nullptr;      // per-front local pivot permutation pool
  int* d_lpos = nullptr;       // and its inverse
  std::vector<int> fidx_static;  // host copy of the static frontIdx pool
  std::vector<long long> fidx_off;
  double* d_Dd = nullptr;
  double* d_Do = nullptr;
  int8_t* d_pk = nullptr;
  std::vector<long long> dpos;
  int* d_maps = nullptr;       // invmap / relmap pool
  symla_gpu::FrontDesc* d_desc = nullptr;
  symla_gpu::ChildLink* d_links = nullptr;
  size_t links_capacity = 0;
  symla_gpu::FrontState* d_state = nullptr;
  symla_gpu::FactorGlobals* d_glob = nullptr;
  int* d_a_colptr = nullptr;
  int* d_a_j = nullptr;
  int* d_a_pos = nullptr;
  int* d_a_idx = nullptr;
  double* d_values = nullptr;
  int* d_sign_final = nullptr;
  double* d_front_delta = nullptr;
  int* d_perm = nullptr;
  // residual
  int* d_rowptr = nullptr;
  int* d_colind = nullptr;
  int* d_vidx = nullptr;
  int* d_srowptr = nullptr;
  int* d_svidx = nullptr;
  // solve workspace
  double* d_W = nullptr;
  int w_nrhs = 0;
  bool w_dirty = true;
  double* d_Bp = nullptr;
  double* d_Z = nullptr;
  double* d_Xf = nullptr;
  double* d_B = nullptr;
  double* d_X = nullptr;
  double* d_R = nullptr;
  double* d_dX = nullptr;
  double* d_Xn = nullptr;
  double* d_Rn = nullptr;
  double* d_norms = nullptr;
  int vec_nrhs = 0;
  double* d_hostvals_tmp = nullptr;
  int* d_scratch_int = nullptr;
  size_t scratch_int_cap = 0;

  // pipelined solve
  int* d_flag_base = nullptr;
  int* d_flags = nullptr;
  int* d_solve_err = nullptr;
  int* d_hflags = nullptr;        // backward helper-part flags (one per slot)
  double* d_hscratch = nullptr;   // backward helper-part partial sums
  int hslot_count = 0;
  int* d_counter = nullptr;  // unfinished-front counter
  int flag_count = 0;
  int solve_epoch = 0;
  int fwd_resident = 0, bwd_resident = 0;
  std::vector<int> solve_np;  // npiv per front the task lists were built for

  // mixed-precision far update workspace (static plan) and error word
  float* d_tcws = nullptr;
  bool tc_static_ready = false;
  int* d_tc_err = nullptr;
  double* d_tc_guard = nullptr;  // growth-guard maxima, 2 per large front of a level
  size_t tc_guard_cap = 0;

  // dynamic (delayed-pivot) allocations for the current factorization
  std::vector<void*> dyn_allocs;
  // front storage allocated by re-planning (pointer, doubles), for the
  // checked build's storage check
  std::vector<std::pair<double*, size_t>> dyn_front_blocks;

  // bounds checks of the checked build: status word (allocated in every
  // build, written only by the checked one) and the front allocations as
  // (lo, hi) pairs on the device
  symla_gpu::CheckWord* d_check = nullptr;
  const double** d_ranges = nullptr;
  size_t ranges_cap = 0;
  std::vector<const double*> h_ranges;

  // bound of every device-side wait on another CTA (solve flags, tensor-core
  // mbarriers), global-timer ns; set by symla_gpu_set_wait_limit_ns
  unsigned long long wait_ns = symla_gpu::kDefaultWaitNs;
  // set when a tensor-core tile's drain ran out: its tensor memory was freed
  // with work possibly outstanding, so no further work is run on the context
  bool unusable = false;

  // GMRES-IR workspace: Krylov vectors (restart + 1) x n x nrhs, a zero
  // column, fixed-order partial sums and per-column coefficients
  double* d_gmres = nullptr;
  size_t gmres_cap = 0;
  double* d_zero = nullptr;
  int zero_len = 0;
  double* d_gpart = nullptr;
  size_t gpart_cap = 0;
  double* d_gcoef = nullptr;
  size_t gcoef_cap = 0;

  // state
  bool factorized = false;
  bool singular = false;
  std::vector<int> singularCols;
  std::vector<symla_gpu::FrontState> hstate;
  symla_factor_info last_info{};
  float phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  cudaEvent_t ev[8] = {};
  double plan_sum_m2 = 0.0;
  int plan_max_m = 0;
  long long nnzL = 0;
  int last_precision = 0;
  int panel_counts[4] = {0, 0, 0, 0};  // large-front panels: speculative full / prefix / failed, sequential
  int seq_dec_counts[4] = {0, 0, 0, 0};  // sequential-path decisions (FactorGlobals::seq_dec)

  // panel kernel choice (the cluster kernel unless SYMLA_PANEL=single)
  bool use_cluster_panel = true;

  // graph launch of the factorization's static pass
  bool use_graph = false;
  cudaGraphExec_t graph_exec = nullptr;
  symla_gpu::KernelOpts graph_ko{};
  int graph_captures = 0, graph_resumes = 0;
  long long graph_kernels = 0;  // kernel nodes of the captured graph (counted per replay)
  // panel iterations per level: the most any factorization of this plan
  // needed (0: within the plan), and the counts the captured graph holds
  std::vector<int> level_iters, graph_level_iters;

  // instrumentation
  bool profiling = false;
  long long launches = 0;
  struct KStat {
    long long launches = 0;
    double ms = 0.0, flops = 0.0, bytes = 0.0;
  } kstat[8];
  // the same per tree level (numLevels x 8, level-major); launches outside a
  // level (permutations, residual) count in kstat only
  std::vector<KStat> level_kstat;
  int cur_level = -1;  // tree level of the launches being issued, or -1
  // large-front panel outcomes per level (profiling, non-graph launches):
  // speculative full / prefix / failed, sequential; numLevels x 4
  std::vector<long long> level_panels;
  struct PendingEv {
    cudaEvent_t a, b;
    int kind, level;
    double flops, bytes;
  };
  std::vector<PendingEv> pending;
  std::vector<cudaEvent_t> evpool;
};
