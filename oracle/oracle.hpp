// ORACLE -- test infrastructure only.
//
// CPU restatement of the reference's numeric factorize / solve / refine path
// (alecjacobson/ma57, "symla"), used only by tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg as the checker. Nothing in the product
// (ma57_b200/) links, imports or calls this code.
//
// It follows, decision for decision:
//   include/symla/dense_kernel.hpp:393-837   DenseLDLT::factor (panel-blocked
//       threshold Bunch-Kaufman, lazy column currency from a per-panel raw
//       snapshot, revert-to-raw, blocked trailing update, re-symmetrize)
//   include/symla/dense_kernel.hpp:919-1059  DenseLDLT::factorStatic
//   include/symla/dense_kernel.hpp:269-297   resymmetrizeTrailingTiled
//   include/symla/multifrontal.hpp:299-805   MultifrontalFactorizer::factorize
//       (extras, front index map, extend, extend-add, kPanelBlockingMinFront,
//       packaging, generated elements, singular roots, OpenMP task DAG)
//   include/symla/solve.hpp:159-508          MultifrontalSolver::solve (serial
//       and task-parallel forward / diagonal / backward)
//   include/symla/refine.hpp:69-144          iterativeRefine
//   include/symla/solver.hpp:140-417         SymLDLT factorize / solve /
//       StaticRegularized retry loop
//   include/symla/parallel/task_graph.hpp    runTaskDag / runTaskDagTopDown
//
// Eigen is not available, so dense products are plain loops (the trailing
// GEMM is a register-blocked kernel in oracle_gemm.cpp). Summation order
// inside products therefore differs from Eigen's; every reference test is
// tolerance based, so parity is judged on inertia, pivot structure where the
// reference pins it, and residuals.
//
// Parity pinning: the reference cannot be compiled in this container (Eigen,
// SuiteSparse AMD and LAPACK are absent), so this restatement is pinned
// against the reference's own known-answer tests, ported in tests/.
#pragma once

#include <cstdint>
#include <vector>

namespace oracle {

struct Inertia {
  int n_pos = 0, n_neg = 0, n_zero = 0;
};

// Column-major dense matrix with explicit leading dimension.
struct MatView {
  double* a = nullptr;
  int rows = 0, cols = 0, ld = 0;
  double& operator()(int i, int j) const { return a[i + static_cast<int64_t>(j) * ld]; }
};

struct Mat {
  int rows = 0, cols = 0;
  std::vector<double> a;
  Mat() = default;
  Mat(int r, int c) : rows(r), cols(c), a(static_cast<size_t>(r) * c, 0.0) {}
  double& operator()(int i, int j) { return a[i + static_cast<size_t>(j) * rows]; }
  double operator()(int i, int j) const { return a[i + static_cast<size_t>(j) * rows]; }
  MatView view() { return MatView{a.data(), rows, cols, rows}; }
};

struct BlockDiagonalD {
  std::vector<double> diag, offdiag;
  void resize(int n) {
    diag.assign(n, 0.0);
    offdiag.assign(n, 0.0);
  }
};

enum class PivotKind { OneByOne = 0, TwoByTwo = 1 };
struct PivotBlock {
  int start;
  PivotKind kind;
};

struct DenseLDLTOptions {
  double pivot_threshold = 0.01;  // accepted and ignored, as in the reference
  double zero_tolerance = 1e-300;
  double relative_pivot_floor = 1e-12;
  int panel_size = 64;
};

struct StaticPivotOptions {
  double delta = 0.0;
  double relative_pivot_floor = 1e-8;
  double absolute_floor = 1e-300;
  int panel_size = 64;
};

struct DenseLDLTResult {
  int n_factored = 0;
  std::vector<int> delayed_cols;
  std::vector<PivotBlock> pivots;
  std::vector<int> perm;
  Inertia inertia;
  double max_growth = 1.0;
  double total_perturbation = 0.0;
  int num_perturbed = 0;
};

DenseLDLTResult denseFactor(MatView A, BlockDiagonalD& D, const DenseLDLTOptions& options, int n_eligible);
DenseLDLTResult denseFactorStatic(MatView A, BlockDiagonalD& D, const StaticPivotOptions& options,
                                  const std::vector<int>& expectedSign, int n_eligible);

// Trailing update C(rows x rows) -= X * Y^T with X, Y rows x p (column-major,
// leading dimensions ldx/ldy); updates the full square. Implemented in
// oracle_gemm.cpp.
void gemmSubNT(int rows, int p, const double* X, int ldx, const double* Y, int ldy, double* C, int ldc);

struct Supernode {
  int firstCol = 0, ncols = 0;
  std::vector<int> rowPattern;
};

struct Symbolic {
  int n = 0;
  std::vector<int> perm;    // final -> original
  std::vector<int> parent;  // etree parent (final order)
  std::vector<Supernode> supernodes;
};

struct Csc {
  int n = 0;
  const int* colptr = nullptr;
  const int* rowind = nullptr;
  const double* vals = nullptr;
};

struct SupernodeFactor {
  std::vector<int> rowIndices;
  int nPivots = 0;
  Mat L;  // m x nPivots
  BlockDiagonalD D;
  std::vector<PivotBlock> pivotBlocks;
  Mat Ltop;  // nPivots x nPivots, d21 slots zeroed
};

struct NumericFactor {
  std::vector<SupernodeFactor> fronts;
  std::vector<int> perm;
  Inertia inertia;
  bool singular = false;
  std::vector<int> singularCols;
  int n = 0;
  double totalPerturbation = 0.0;
  int numPerturbed = 0;
  int numDelayedColumns = 0;  // extras summed over fronts (diagnostic)
  std::vector<int> parentSN;
  std::vector<std::vector<int>> childrenSN;
  std::vector<int> rootsSN;
};

struct MultifrontalOptions {
  bool parallel = false;
  int num_threads = 0;
  long long task_cutoff = -1;
  bool static_pivoting = false;
  StaticPivotOptions staticOptions;
  std::vector<int> expectedSign;  // final order
};

NumericFactor multifrontalFactorize(const Symbolic& sf, const Csc& A, const DenseLDLTOptions& options,
                                    const MultifrontalOptions& mfOptions);

struct SolveOptions {
  bool parallel = false;
  int num_threads = 0;
  long long task_cutoff = -1;
};

// B, result: n x nrhs column-major.
Mat multifrontalSolve(const NumericFactor& nf, const Mat& B, const SolveOptions& opts);

struct RefinementOptions {
  int max_iterations = 10;
  double tolerance = 1e-14;
};
struct RefinementResult {
  int iterations = 0;
  double initial_relative_residual = 0.0;
  double final_relative_residual = 0.0;
};

double sparseMaxAbsRowSum(const Csc& A);
// R = B - sym(A_lower) * X  (selfadjointView<Lower>)
void symLowerResidual(const Csc& A, const Mat& X, const Mat& B, Mat& R);

enum class Mode { ThresholdPivot = 0, StaticRegularized = 1 };

// Mirror of symla::SymLDLT<double> (solver.hpp:29-418) over a precomputed
// symbolic analysis.
class SymLDLT {
 public:
  Mode mode = Mode::ThresholdPivot;
  double pivot_threshold = 0.01;
  bool parallel = true;
  int num_threads = 0;
  bool use_kkt_blocks = false;
  int kkt_n1 = 0, kkt_n2 = 0;
  bool use_explicit_signs = false;
  std::vector<int> expected_signs_orig;
  double initial_regularization_delta = 0.0;
  int max_regularization_retries = 10;
  double regularization_growth = 10.0;
  double static_pivot_relative_floor = 1e-8;
  double static_pivot_absolute_floor = 1e-300;
  // dense-kernel knobs the tests reach (defaults = reference defaults)
  double zero_tolerance = 1e-300;
  double relative_pivot_floor = 1e-12;

  double last_regularization_delta = 0.0;
  int regularization_retries_used = 0;
  bool factorized = false;
  Inertia inertia;
  Symbolic symbolic;
  NumericFactor numeric;
  std::vector<double> attemptDeltas;  // every delta tried in the last factorize()
  std::vector<int> attemptOk;

  void setSymbolic(Symbolic s) {
    symbolic = std::move(s);
    factorized = false;
  }
  // Throws std::logic_error / std::invalid_argument / std::runtime_error
  // exactly where the reference does.
  void factorize(const Csc& A);
  Mat solve(const Mat& B) const;
  RefinementResult solveWithRefinement(const Csc& A, const Mat& B, Mat& X, const RefinementOptions& o) const;

 private:
  std::vector<int> buildExpectedSignOriginal(int n) const;
  void factorizeStaticRegularized(const Csc& A);
};

}  // namespace oracle
