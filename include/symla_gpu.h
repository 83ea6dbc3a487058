/*
 * symla_gpu.h -- C ABI of the B200 numeric factorize / solve path of symla.
 *
 * The reference library (alecjacobson/ma57, "symla") is a header-only C++
 * template library; its numeric work happens behind two static template
 * seams that SymLDLT<double> calls:
 *
 *   MultifrontalFactorizer<double>::factorize(sf, A, opts, mfOpts) -> NumericFactor
 *       include/symla/multifrontal.hpp:299-300 (called from solver.hpp:158, :379)
 *   MultifrontalSolver<double>::solve(nf, B, solveOpts) -> DenseMatrix
 *       include/symla/solve.hpp:159 (called from solver.hpp:217)
 *
 * plus the residual of iterativeRefine (refine.hpp:97-144, called from
 * solver.hpp:238). The entry points below replace those seams: plain pointers
 * and sizes, int status codes, no C++ or torch types. The symbolic analysis
 * (ordering, elimination tree, supernodes; symbolic.hpp:195-399) stays on the
 * host; symla_analyze() is a restatement of it that produces the same
 * structure, for callers that do not run the reference's own analysis.
 *
 * Conventions
 *   - Matrices are CSC, 0-based, int32 indices (Eigen::SparseMatrix<double,
 *     ColMajor, int> in compressed mode). Only the lower triangle (row >= col)
 *     of the values is read (multifrontal.hpp:190-216, refine.hpp:88-92).
 *   - Dense right-hand sides are column-major with a leading dimension.
 *   - Every call that takes a `*_on_device` flag accepts host pointers (0) or
 *     device pointers on the context's GPU (1).
 *   - A context owns its device memory and one CUDA stream; it is not
 *     thread-safe (same contract as the reference's SymLDLT).
 *   - On error the status is returned and symla_last_error() holds a message
 *     for the calling thread.
 */
#ifndef SYMLA_GPU_H_
#define SYMLA_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The C++ wrapper maps them onto the reference's exceptions:
 * NOT_ANALYZED/NOT_FACTORIZED/SINGULAR -> std::logic_error
 * (solver.hpp:141-143, :199-206), BAD_SIZE/INVALID -> std::invalid_argument
 * (solver.hpp:55, :207-209, :301-311), RETRY_EXHAUSTED -> std::runtime_error
 * (solver.hpp:403-413). */
enum {
  SYMLA_OK = 0,
  SYMLA_ERR_NOT_ANALYZED = 1,
  SYMLA_ERR_NOT_FACTORIZED = 2,
  SYMLA_ERR_SINGULAR = 3,
  SYMLA_ERR_BAD_SIZE = 4,
  SYMLA_ERR_RETRY_EXHAUSTED = 5,
  SYMLA_ERR_OOM = 6,
  SYMLA_ERR_TIMEOUT = 7,
  SYMLA_ERR_CUDA = 8,
  SYMLA_ERR_INVALID = 9,
  SYMLA_ERR_NO_DEVICE = 10,
  SYMLA_ERR_INTERNAL = 11
};

/* Orderings (OrderingType, ordering.hpp:31-35). SYMLA_ORDER_METIS takes
 * METIS_NodeND's first output array, which lists the original vertex placed
 * at each new position: the nested-dissection pivot order. The reference
 * takes the second array instead (ordering.hpp:130-141), which is the inverse
 * of that permutation; SYMLA_ORDER_METIS_IPERM reproduces the reference's
 * permutation exactly, for callers that need bit-identical symbolic results
 * with it. The two agree on AMD and Natural. */
enum { SYMLA_ORDER_AMD = 0, SYMLA_ORDER_METIS = 1, SYMLA_ORDER_NATURAL = 2, SYMLA_ORDER_METIS_IPERM = 3 };
enum { SYMLA_MODE_THRESHOLD = 0, SYMLA_MODE_STATIC = 1 };
/* Arithmetic of the Schur-complement (trailing) updates of large fronts.
 * Pivot tests, D, 2x2 inversion, L, the solves and the refinement residual
 * are FP64 in both. */
enum { SYMLA_PREC_FP64 = 0, SYMLA_PREC_MIXED = 1 };

/* Thread-local message for the most recent failing call on this thread. */
const char* symla_last_error(void);

/* ------------------------------------------------------------------ */
/* Host symbolic analysis (replaces SymbolicFactor::analyze,           */
/* symbolic.hpp:195-399, for callers without the reference's analysis) */
/* ------------------------------------------------------------------ */
typedef struct symla_symbolic symla_symbolic;

typedef struct {
  int n;
  int num_supernodes;
  int num_fundamental;
  int64_t pattern_len;        /* sum of supernode rowPattern sizes */
  int64_t fundamental_len;    /* sum of fundamental rowPattern sizes */
  int64_t storage_nnz;        /* sum of Supernode::storageNnz() */
} symla_symbolic_info;

/* SymLDLT::analyzePattern (solver.hpp:133-137) with SymbolicFactorOptions
 * {max_relax_size, max_relax_fill_fraction} (symbolic.hpp:161-184). */
int symla_analyze(int n, const int* colptr, const int* rowind, int ordering, int max_relax_size,
                  double max_relax_fill_fraction, symla_symbolic** out);
void symla_symbolic_destroy(symla_symbolic* sym);
/* computeOrdering (ordering.hpp:84-149) alone: perm[k] = original index of
 * the k-th pivot, before the elimination-tree postorder that symla_analyze
 * applies on top of it (symbolic.hpp:207-218). Either triangle or both may be
 * stored. */
int symla_compute_ordering(int n, const int* colptr, const int* rowind, int ordering, int* perm);
int symla_symbolic_get_info(const symla_symbolic* sym, symla_symbolic_info* info);
/* Any output pointer may be NULL. perm/etree_parent/etree_colcount: n.
 * sn_first/sn_ncols: num_supernodes; sn_ptr: num_supernodes+1;
 * sn_rows: pattern_len (supernode si's rowPattern is
 * sn_rows[sn_ptr[si] .. sn_ptr[si+1])). */
int symla_symbolic_get(const symla_symbolic* sym, int* perm, int* etree_parent, int* etree_colcount, int* sn_first,
                       int* sn_ncols, int* sn_ptr, int* sn_rows);
/* The fundamental (pre-amalgamation) supernodes (SymbolicFactor::
 * fundamentalSupernodes), same layout, num_fundamental entries. */
int symla_symbolic_get_fundamental(const symla_symbolic* sym, int* sn_first, int* sn_ncols, int* sn_ptr,
                                   int* sn_rows);
/* Build a symbolic handle from a caller's own analysis (for a maintainer
 * whose SymLDLT keeps the reference's SymbolicFactor): perm, etree parent,
 * and the final supernodes. */
int symla_symbolic_import(int n, const int* perm, const int* etree_parent, int num_supernodes, const int* sn_first,
                          const int* sn_ncols, const int* sn_ptr, const int* sn_rows, symla_symbolic** out);

/* ------------------------------------------------------------------ */
/* Device context                                                      */
/* ------------------------------------------------------------------ */
typedef struct symla_gpu_ctx symla_gpu_ctx;

/* Uploads the symbolic structure and precomputes, once per pattern, the
 * A-value -> front scatter map, child -> parent extend-add maps, the level
 * schedule and the front arena layout. `colptr/rowind` is the pattern the
 * values of later factorize calls will follow (refactorize reuses it). */
int symla_gpu_create(const symla_symbolic* sym, int n, const int* colptr, const int* rowind, int device,
                     symla_gpu_ctx** out);
void symla_gpu_destroy(symla_gpu_ctx* ctx);

typedef struct {
  int mode;                     /* SYMLA_MODE_* */
  int precision;                /* SYMLA_PREC_* */
  double pivot_threshold;       /* u; accepted and ignored (dense_kernel.hpp:57-69) */
  double zero_tolerance;        /* default 1e-300 (dense_kernel.hpp:77) */
  double relative_pivot_floor;  /* default 1e-12 (dense_kernel.hpp:102) */
  /* Mode::StaticRegularized, one attempt (dense_kernel.hpp:227-253) */
  double static_delta;          /* <= 0: sqrt(eps) * front max, per front */
  double static_rel_floor;      /* default 1e-8 */
  double static_abs_floor;      /* default 1e-300 */
  const int* expected_sign;     /* n entries in ORIGINAL index space, or NULL */
  const double* front_delta;    /* optional per-supernode delta override (learned), or NULL */
} symla_factor_opts;

void symla_factor_opts_default(symla_factor_opts* o);

typedef struct {
  int n_pos, n_neg, n_zero;
  int singular;                 /* NumericFactor::singular */
  int n_singular;               /* size of singularCols */
  int num_perturbed;
  double total_perturbation;
  int num_delayed;              /* columns that arrived as extras at some front */
  int used_dynamic_path;        /* delays forced the re-planned (host-synchronised) path */
  double max_growth;
  float factor_ms;              /* device time of the factorization (CUDA events) */
} symla_factor_info;

/* MultifrontalFactorizer::factorize for one attempt (ThresholdPivot, or one
 * StaticRegularized pass with a fixed delta). values: nnz entries in the
 * CSC order given at create time. */
int symla_gpu_factorize(symla_gpu_ctx* ctx, const double* values, int values_on_device, const symla_factor_opts* opts,
                        symla_factor_info* info);

/* SymLDLT::factorizeStaticRegularized's inertia-controlled retry loop
 * (solver.hpp:328-417) driving symla_gpu_factorize. expected_sign (original
 * index space, n entries) or kkt_n1/kkt_n2 (>= 0) describe the expectation;
 * with neither, one pass and no check. Returns SYMLA_ERR_RETRY_EXHAUSTED
 * when the budget runs out. */
typedef struct {
  double initial_delta;         /* <= 0: sqrt(eps) * max|A| */
  int max_retries;              /* default 10 */
  double growth;                /* default 10 */
  double static_rel_floor;
  double static_abs_floor;
  const int* expected_sign;     /* original index space, or NULL */
  int kkt_n1, kkt_n2;           /* used when expected_sign is NULL and kkt_n1 >= 0 */
  int precision;
  const double* front_delta;    /* optional per-supernode first-attempt deltas (learned); when
                                   that attempt fails, the escalation resumes one growth step
                                   above max(initial delta, smallest front delta) */
} symla_regularize_opts;

void symla_regularize_opts_default(symla_regularize_opts* o);

typedef struct {
  int retries_used;
  double last_delta;
  int attempts;
  double attempt_delta[32];
  int attempt_ok[32];
} symla_regularize_info;

int symla_gpu_factorize_regularized(symla_gpu_ctx* ctx, const double* values, int values_on_device,
                                    const symla_regularize_opts* opts, symla_factor_info* info,
                                    symla_regularize_info* rinfo);

/* MultifrontalSolver::solve: X = A^{-1} B, B and X n x nrhs column-major.
 * Fails with SYMLA_ERR_NOT_FACTORIZED / SYMLA_ERR_SINGULAR like
 * SymLDLT::solve (solver.hpp:198-218). */
int symla_gpu_solve(symla_gpu_ctx* ctx, const double* B, int ldb, int nrhs, double* X, int ldx, int on_device);

typedef struct {
  int iterations;
  double initial_relative_residual;
  double final_relative_residual;
} symla_refine_info;

/* solve + iterativeRefine (refine.hpp:97-144) against the values of the
 * matrix (same pattern as at create time), FP64 residual on the device. */
int symla_gpu_solve_refine(symla_gpu_ctx* ctx, const double* values, const double* B, int ldb, int nrhs, double* X,
                           int ldx, int on_device, int max_iterations, double tolerance, symla_refine_info* info);

/* GMRES-IR (no counterpart in the reference; refine.hpp:52-57 records
 * fixed-precision refinement as its limitation): refinement on the FP64
 * residual with iterativeRefine's stopping and acceptance rules, each
 * correction solved by restarted GMRES (`restart` in [1, 64] Krylov vectors
 * per outer step) preconditioned by the device LDL^T solve. It converges
 * where fixed-precision refinement stagnates with a factor that is only an
 * approximate inverse: the mixed-precision factorization, or a static-pivot
 * factorization with large perturbations. Keeps (restart + 1) x n x nrhs
 * doubles of Krylov vectors on the device. */
typedef struct {
  int outer_iterations;
  int inner_iterations;         /* GMRES steps over all outer iterations (one solve + one SpMV each) */
  double initial_relative_residual;
  double final_relative_residual;
} symla_gmres_info;

int symla_gpu_solve_gmres_refine(symla_gpu_ctx* ctx, const double* values, const double* B, int ldb, int nrhs,
                                 double* X, int ldx, int on_device, int max_outer, int restart, double tolerance,
                                 symla_gmres_info* info);

/* Final-order indices of the columns that could not be pivoted anywhere
 * (NumericFactor::singularCols, sorted). Returns the count; writes at most
 * cap entries. */
int symla_gpu_singular_cols(symla_gpu_ctx* ctx, int* cols, int cap);

/* Per-front factor export (NumericFactor::fronts[si], multifrontal.hpp:118-135):
 * sizes first, then contents. rowIndices: m; L: m x npiv column-major (the
 * strictly lower part of the top npiv x npiv block and the rows below it are
 * multipliers; the (k+1,k) slot of a 2x2 block holds d21); d_diag/d_off:
 * npiv; piv_start/piv_kind: number of pivot blocks (returned). */
int symla_gpu_num_fronts(symla_gpu_ctx* ctx);
int symla_gpu_front_size(symla_gpu_ctx* ctx, int si, int* m, int* npiv);
int symla_gpu_front_get(symla_gpu_ctx* ctx, int si, int* row_indices, double* L, double* d_diag, double* d_off,
                        int* piv_start, int* piv_kind);

/* The context's CUDA stream (cudaStream_t), for callers that time or order
 * work around the library. */
void* symla_gpu_stream(symla_gpu_ctx* ctx);

/* Device time of the phases of the most recent factorize / solve calls
 * (CUDA events): [0] assembly, [1] dense factorization, [2] trailing update,
 * [3] forward+diagonal solve, [4] backward solve, [5] residual, [6] total
 * factorize, [7] total solve. */
int symla_gpu_phase_ms(symla_gpu_ctx* ctx, float* ms, int cap);

/* Kernel instrumentation. When enabled, every launch of the library's
 * kernels is bracketed by CUDA events on the context's stream; per kernel
 * kind the launch count, summed device time and algorithmic work are kept
 * until reset. Kinds: 0 far (deferred, outer-block) Schur-complement update
 * (with FP64 precision the near updates run in the same launch and count
 * here),
 * 1 panel factorization, 2 small-front kernel, 3 assembly, 4 forward solve,
 * 5 backward solve, 6 residual, 7 near (in-block) Schur-complement update.
 * out[0] launches, out[1] total ms, out[2] algorithmic flops, out[3]
 * algorithmic bytes. */
enum { SYMLA_KERNEL_TRAILING = 0, SYMLA_KERNEL_PANEL = 1, SYMLA_KERNEL_SMALL = 2, SYMLA_KERNEL_ASSEMBLE = 3,
       SYMLA_KERNEL_FORWARD = 4, SYMLA_KERNEL_BACKWARD = 5, SYMLA_KERNEL_RESIDUAL = 6, SYMLA_KERNEL_NEAR = 7,
       SYMLA_KERNEL_KINDS = 8 };
int symla_gpu_set_profiling(symla_gpu_ctx* ctx, int enable);

/* Failure handling (no reference counterpart; the reference has no device
 * waits or device memory).
 *
 * symla_gpu_set_wait_limit_ns: every device-side wait on another CTA's
 * progress -- the pipelined solves' block flags and the tensor-core Schur
 * update's copy/MMA barriers -- gives up after `ns` nanoseconds of the GPU's
 * global timer (0 restores the default of 2 s). A wait that runs out makes
 * the call return SYMLA_ERR_TIMEOUT; the context stays usable (a solve can be
 * repeated, a factorization must be repeated). If a tensor-core tile that
 * gave up cannot then confirm, within the default limit, that its copies and
 * MMAs have finished, the call also reports SYMLA_ERR_TIMEOUT and every later
 * call on the context fails with SYMLA_ERR_CUDA: destroy it.
 *
 * symla_gpu_set_memory_limit: process-wide cap, in bytes, on the device
 * memory that each later symla_gpu_create may allocate for a context's plan
 * (front arena, maps, solve workspaces); 0 removes it. A plan that does not
 * fit fails with SYMLA_ERR_OOM before touching the GPU further, like a
 * failing cudaMalloc does without a cap. */
int symla_gpu_set_wait_limit_ns(symla_gpu_ctx* ctx, unsigned long long ns);
int symla_gpu_set_memory_limit(long long bytes);

/* Graph launch of the factorization (no reference counterpart): when
 * enabled (and profiling is off), the static pass over all tree levels, with
 * a few spare panel iterations per level, is captured once per set of
 * factorization options into a CUDA graph and replayed by every later
 * factorize; a level that its planned iterations did not finish (or a
 * delayed pivot) is continued on the host exactly as without the graph.
 * graph_stats: captures made and factorizations that needed that host
 * continuation. */
int symla_gpu_set_graph(symla_gpu_ctx* ctx, int enable);

/* Tile schedule per tree level (no reference counterpart; chosen by the
 * autotuner in ma57_b200/autotune.py). level_info: out6 = {small fronts,
 * their max m, large fronts, their max m, small-front kernel threads, panel
 * cluster CTAs}. set_level_schedule: small-front kernel threads in {32
 * (one warp per front, eight fronts per CTA; fronts of at most 32 rows),
 * 128, 256} and panel cluster size in {2, 4, 8, 16}, or 1 for the single-CTA
 * panel kernel (no cluster barriers: faster for levels whose panels decide
 * many pivots one at a time), 0 = chosen by front size; a cluster size too
 * small for the level's fronts falls back to the default. */
int symla_gpu_level_info(symla_gpu_ctx* ctx, int level, int* out6);
int symla_gpu_set_level_schedule(symla_gpu_ctx* ctx, int level, int small_threads, int cluster_ctas);
/* Rows per tile of the level's Schur-complement update (the tile shape
 * rows x 64): 128, or 64 for levels of small fronts; 0 = 128. */
int symla_gpu_set_level_update_rows(symla_gpu_ctx* ctx, int level, int rows);
int symla_gpu_level_update_rows(symla_gpu_ctx* ctx, int level, int* rows);
int symla_gpu_graph_stats(symla_gpu_ctx* ctx, int* captures, int* resumes);
int symla_gpu_kernel_stats(symla_gpu_ctx* ctx, int kind, double* out4);
/* The same per tree level (the per-phase timers the reference keeps under
 * SYMLA_PROFILE, multifrontal.hpp:56-78, by level instead of by phase):
 * launches of `kind` issued for that level's fronts (factorization) or
 * blocks (solves). Algorithmic flops of the Schur updates are counted on the
 * device per factorization, not per level, and read 0 here. */
int symla_gpu_level_kernel_stats(symla_gpu_ctx* ctx, int level, int kind, double* out4);
/* Large-front panel outcomes of a level, counted while profiling is enabled
 * (ordinary launches, not the graph): [0] speculated and accepted whole,
 * [1] accepted up to a failing pivot, [2] failed at the first pivot, [3] run
 * sequentially throughout (the totals of symla_gpu_plan_stats [7..10]). */
int symla_gpu_level_panel_stats(symla_gpu_ctx* ctx, int level, long long* out4);
void symla_gpu_reset_kernel_stats(symla_gpu_ctx* ctx);
/* Number of kernels the library launched since the last reset (the kernel
 * nodes of a replayed factorization graph count at every replay). */
long long symla_gpu_launch_count(symla_gpu_ctx* ctx);

/* Front-size statistics of the plan: [0] fronts, [1] levels, [2] max m,
 * [3] sum m^2, [4] algorithmic factorization flops of the last factorize
 * (lower-triangle convention), [5] nnz(L) entries, [6] arena doubles;
 * large-front panels of the last factorize: [7] speculated and accepted
 * whole, [8] accepted up to a failing pivot, [9] failed at the first pivot
 * (one sequential decision), [10] run sequentially throughout; decisions of
 * the panels' sequential (per-pivot) path: [11] 1x1 at k by the first
 * Bunch-Kaufman test or an isolated column, [12] 1x1 at k by the sigma test,
 * [13] interchange then 1x1, [14] 2x2. Returns the number of entries (15). */
int symla_gpu_plan_stats(symla_gpu_ctx* ctx, double* out, int cap);

/* Learned first-attempt delta for Mode::StaticRegularized (no reference
 * counterpart; the reference starts every factorization's escalation from
 * the same delta, solver.hpp:328-417). A multilayer perceptron maps
 * SYMLA_MLP_INPUTS standardised per-front statistics to the front's
 * first-attempt delta in decades above the plain first attempt
 * (symla_regularize_opts.front_delta), trained on the GPU from the deltas
 * the escalation loop itself accepted; on an inertia failure the plain
 * escalation resumes above the failed attempt. FP64; parameters in
 * the order W1 (H x IN, row-major), b1 (H), W2 (H x H), b2 (H), w3 (H), b3. */
#define SYMLA_MLP_INPUTS 8
#define SYMLA_MLP_HIDDEN 32
#define SYMLA_MLP_PARAMS (SYMLA_MLP_HIDDEN * SYMLA_MLP_INPUTS + SYMLA_MLP_HIDDEN + SYMLA_MLP_HIDDEN * SYMLA_MLP_HIDDEN + \
                          SYMLA_MLP_HIDDEN + SYMLA_MLP_HIDDEN + 1)
typedef struct symla_mlp symla_mlp;
int symla_mlp_create(int device, const double* params, symla_mlp** out);
void symla_mlp_destroy(symla_mlp* mlp);
int symla_mlp_get_params(symla_mlp* mlp, double* params_out);
/* Y[s] = network(X[s, :]) for B samples (X row-major B x SYMLA_MLP_INPUTS, host). */
int symla_mlp_predict(symla_mlp* mlp, const double* X, int B, double* Y);
/* Gradient of the mean squared error (1/B) sum (Y - T)^2 w.r.t. the
 * parameters, and that error, at the current parameters. */
int symla_mlp_gradient(symla_mlp* mlp, const double* X, const double* T, int B, double* grad, double* loss);
/* Adam (beta 0.9 / 0.999) over `epochs` passes of minibatches (<= 0: full
 * batch); final_loss (optional) = mean squared error after training. */
int symla_mlp_train(symla_mlp* mlp, const double* X, const double* T, int B, int epochs, int minibatch, double lr,
                    double* final_loss);

/* Relative residual ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf) of
 * a device-resident candidate solution X against device-resident B
 * (column-major, n x nrhs, leading dimensions ldx, ldb >= n), for the matrix
 * of the last factorization; *rel_residual receives it on the host. It is
 * the measure symla_gpu_solve_refine reports, computed without allocating
 * any device memory: for callers whose device memory is owned by another
 * allocator, or whose loop cannot take the device-wide synchronisation of
 * cudaMalloc / cudaFree. This entry point has no counterpart in the
 * reference.
 *
 * Its scratch (the residual and four norm accumulators) is one fixed
 * device array inside the library, of SYMLA_NOALLOC_RESIDUAL_MAX_ENTRIES
 * doubles plus 256 bytes, present on every GPU that loads the library until
 * the process exits. n * nrhs above that maximum is rejected with
 * SYMLA_ERR_BAD_SIZE. The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that
 * first call before any stream capture. Every call uses the same array and
 * clears the accumulators it needs at its start, so calls whose work
 * overlaps on the GPU (from several threads, contexts or streams) race and
 * must be serialised by the caller. Runs on the context's stream and
 * returns after it synchronises. That stream does not synchronise with the
 * legacy default stream or any other stream: X and B must be complete
 * before the call (synchronise their producer, or record an event after it
 * and make symla_gpu_stream(ctx) wait on it). The array's device address is
 * looked up on a device's first call and kept; a cudaDeviceReset of that
 * device afterwards is not supported. */
#define SYMLA_NOALLOC_RESIDUAL_MAX_ENTRIES (1 << 20)
int symla_gpu_relative_residual_noalloc(symla_gpu_ctx* ctx, const double* X, int ldx, const double* B, int ldb,
                                        int nrhs, double* rel_residual);

/* Bounds-checked build (libsymla_b200_checked.so, compiled with
 * -DSYMLA_GPU_CHECKED; same entry points). Before and after every
 * factorization and before every solve it validates the device tables
 * (front descriptors and their storage, row indices, extend-add maps, A's
 * scatter map, pivot counts, solve workspace slices), and inside the kernels
 * every access whose index comes from a table is checked before it is made.
 * A failed check skips the access and records the first failure in a status
 * word on the device; the call then returns SYMLA_ERR_INTERNAL naming it, and
 * every later call on the context fails with SYMLA_ERR_CUDA. No check traps
 * or asserts. No counterpart in the reference (its opt-in sanitizer builds
 * are CPU-side, test/CMakeLists.txt:141-149).
 *
 * symla_gpu_checked_build: 1 in the checked build, 0 in the ordinary one.
 * symla_gpu_check_status: the status word (failed checks so far, the first
 * one's code, the front or entry where it happened); always zero in the
 * ordinary build. Codes: 1 descriptor shape, 2 front storage, 3 row index,
 * 4 child link, 5 parent-to-child map, 6 child-to-parent map, 7 A scatter
 * entry, 8 pivot count, 9 contribution-block read, 10 solve permutation,
 * 11 level-solve row, 12 solve workspace. */
int symla_gpu_checked_build(void);
int symla_gpu_check_status(symla_gpu_ctx* ctx, int* count, int* code, long long* where);

#ifdef __cplusplus
}
#endif

#endif /* SYMLA_GPU_H_ */
