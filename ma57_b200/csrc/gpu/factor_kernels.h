// Host launchers for the factorization and solve kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace symla_gpu {

// Fronts whose m is at most this go through the one-CTA shared-memory kernel.
constexpr int kSmallFrontMax = 128;
// Panel width of the large-front path.
constexpr int kPanelWidth = 32;
// Rows of one assembly task when a level's (front, 32 columns) tasks are
// too few to fill the GPU (they are then split into row chunks).
constexpr int kAsmRows = 1024;

cudaError_t configure_factor_kernels();
size_t small_front_smem(int m);

// tasks: (front, first column, first row, end row or -1 for the front's m)
void launch_assemble(const FrontDesc* fronts, const ChildLink* links, FrontState* st, const int* tasks,
                     int ntasks, const int* a_colptr, const KernelOpts& o, const FactorGlobals* g, int level,
                     int dynamic, cudaStream_t stream);
void launch_factor_small(const FrontDesc* fronts, const ChildLink* links, FrontState* st, const int* list, int count,
                         int max_m, const int* a_colptr, const KernelOpts& o, FactorGlobals* g, int level, int dynamic,
                         cudaStream_t stream, int threads = 0);  // threads: 32 (a warp per front, fronts of
                                                                 // <= 32 rows), 128, 256, or 0 (by front size)
// Single-CTA panel kernel. Its two working columns (2 m doubles per front)
// live in shared memory when panel_fits_shared(max_m), else in `cols`
// (device, 2 max_m doubles per front of the list), which is then required.
bool panel_fits_shared(int max_m);
cudaError_t launch_panel(const FrontDesc* fronts, FrontState* st, const int* list, int count, int max_m, int nb,
                         const KernelOpts& o, FactorGlobals* g, int level, int dynamic, cudaStream_t stream,
                         double* cols);
// Cluster panel (panel_cluster.cu): returns 0 from cluster_size_for when a
// front is too large for it with nb-pivot panels (the single-CTA panel
// kernel then runs).
int cluster_size_for(int max_m, int count, int nb = kPanelWidth);
// whether a cluster of cs CTAs (2, 4, 8 or 16) can hold fronts of max_m rows
// with nb-pivot panels
bool cluster_size_fits(int max_m, int cs, int nb = kPanelWidth);
// Pivots per panel for a level whose tallest large front has max_m rows:
// kPanelWidth when a cluster holds such fronts at that width, else the widest
// panel (at least 8 pivots) a 16-CTA cluster holds, else kPanelWidth for the
// single-CTA kernel.
int panel_width_for(int max_m, int count);
cudaError_t configure_cluster_panel();
// cs: 2, 4, 8 or 16, or 0 for cluster_size_for's choice
cudaError_t launch_cluster_panel(const FrontDesc* fronts, FrontState* st, const int* list, int count, int max_m,
                                 int nb, const KernelOpts& o, FactorGlobals* g, int level, int dynamic,
                                 cudaStream_t stream, int cs = 0);
// Mixed-precision far update (schur_tc.cu): TF32x3 tcgen05 GEMM fed by TMA.
size_t tc_far_smem();
cudaError_t configure_tc_far();
int tc_max_fronts();
// guard: 2 doubles per list entry, zeroed before launch_tc_split (max|L|, max|L D|)
void launch_tc_split(const FrontDesc* fronts, const FrontState* st, const int* list, int count, float* const* ws,
                     double* guard, int max_m, const FactorGlobals* g, int level, int dynamic, cudaStream_t stream);
void launch_tc_far(const FrontDesc* fronts, FrontState* st, const int* list, int count, const CUtensorMap* maps,
                   const double* guard, int grid, FactorGlobals* g, int level, int dynamic, int* err,
                   cudaStream_t stream);

// Checked build: validate the tables of `count` fronts (list, or all fronts
// when list is null) into o.chk. ranges: device array of nranges (lo, hi)
// pairs, the front allocations; phase 0 before the factorization, 1 after
// it, 2 before a solve (W slices of wcols columns inside [wlo, whi)).
void launch_validate_fronts(const FrontDesc* fronts, const ChildLink* links, const FrontState* st, const int* list,
                            int count, int num_fronts, int n, const int* a_colptr, const KernelOpts& o,
                            const double* const* ranges, int nranges, const double* wlo, const double* whi,
                            int wcols, int phase, cudaStream_t stream);

// graph launches: atomicMin(g->unfinished_level, level) if a front of the
// list is not finished
void launch_mark_unfinished(const FrontState* st, const int* list, int count, FactorGlobals* g, int level,
                            cudaStream_t stream);
// *out += number of fronts in list not yet finished (flag kFlagDone unset)
void launch_count_unfinished(const FrontState* st, const int* list, int count, int* out, cudaStream_t stream);
// near (far = false) / far (far = true) Schur-complement update, FP64. With
// tc_guard (far only; the split pre-pass's maxima, 2 per list entry) it
// applies just the blocks that tc_block_ok sends away from the tensor cores.
// tile_rows: 128 (default) or 64 rows per update tile.
void launch_update(bool far, const FrontDesc* fronts, FrontState* st, const int* list, int count, int grid_x,
                   FactorGlobals* g, int level, int dynamic, cudaStream_t stream, const double* tc_guard = nullptr,
                   int tile_rows = 128);
// near and far updates of every front in one launch (FP64 path)
void launch_update_both(const FrontDesc* fronts, FrontState* st, const int* list, int count, int grid_x,
                        FactorGlobals* g, int level, int dynamic, cudaStream_t stream, int tile_rows = 128);

// Solve
// chk: status word of the checked build's permutation-entry checks (or null)
void launch_permute_in(int n, int nrhs, const int* perm, const double* B, int ldb, double* Bp, cudaStream_t stream,
                       CheckWord* chk = nullptr);
void launch_permute_out(int n, int nrhs, const int* perm, const double* X, double* Xout, int ldx, cudaStream_t stream,
                        CheckWord* chk = nullptr);
// Pipelined level solves (one cooperative launch per level; see
// solve_kernels.cu). tasks: int4 (see the kernels); flags indexed by
// flag_base[front] + block, compared against epoch; every wait on another
// CTA's flag gives up after wait_ns of the global timer (error word set).
int solve_block_rows();
int solve_rhs_chunk();
cudaError_t solve_max_resident(int device, int* fwd_ctas, int* bwd_ctas);
cudaError_t launch_forward_pipelined(const FrontDesc* fronts, const ChildLink* links, const FrontState* st,
                                     const int4* tasks, int ntasks, int grid, const int* flag_base, int* flags,
                                     int epoch, int* err, unsigned long long wait_ns, int nrhs, int c0,
                                     const double* Bp, int n, cudaStream_t stream);
cudaError_t launch_backward_pipelined(const FrontDesc* fronts, const FrontState* st, const int4* tasks, int ntasks,
                                      int grid, const int* flag_base, int* flags, int* hflags, double* hscratch,
                                      int epoch, int* err, unsigned long long wait_ns, int nrhs, int c0, double* X,
                                      int n, cudaStream_t stream);

// Residual R = B - sym(A) X in the original index space (full symmetric CSR
// gathered from the stored lower triangle); rowptr/colind/vidx describe it.
void launch_residual(int n, int nrhs, const int* rowptr, const int* colind, const int* vidx, const double* vals,
                     const double* X, int ldx, const double* B, int ldb, double* R, cudaStream_t stream);
// out[slot] = max(out[slot], max |v|) over len entries (out pre-zeroed).
void launch_absmax(const double* v, long long len, double* out, cudaStream_t stream);
// Max absolute row sum over the stored entries (refine.hpp:69-81).
void launch_rowsum_max(int n, const int* srowptr, const int* svidx, const double* vals, double* out,
                       cudaStream_t stream);
// X += dX (len entries)
void launch_axpy(long long len, const double* dx, double* x, cudaStream_t stream);
void launch_copy2d(int rows, int cols, const double* src, int lds, double* dst, int ldd, cudaStream_t stream);
// GMRES-IR vector work over all right-hand sides at once; vector i, column c
// at V + i * vs + c * n. multi_dot writes nvec x nrhs x multi_dot_blocks(n)
// fixed-order partial sums of V_i[:, c] . W[:, c]; multi_axpy: W[:, c] -=
// sum_i coef[i nrhs + c] V_i[:, c]; col_scale: Y[:, c] = alpha[c] X[:, c].
int multi_dot_blocks(int n);
void launch_multi_dot(int n, int nrhs, int nvec, const double* V, long long vs, const double* W, double* partial,
                      cudaStream_t stream);
void launch_multi_axpy(int n, int nrhs, int nvec, const double* V, long long vs, const double* coef, double* W,
                       cudaStream_t stream);
void launch_col_scale(int n, int nrhs, const double* alpha, const double* X, double* Y, cudaStream_t stream);

}  // namespace symla_gpu
