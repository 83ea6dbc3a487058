/*
 * symla_gpu_backend.hpp -- the C++ binding a symla maintainer adds so that
 * SymLDLT<double> runs its numeric work on the B200 path.
 *
 * The reference keeps SymLDLT's code and swaps its two static template
 * seams (include/symla/multifrontal.hpp:299-300 and include/symla/solve.hpp:159)
 * for the calls below; the binding keeps one Backend next to the
 * SymbolicFactor it analysed. It is header-only over include/symla_gpu.h and
 * generic in the reference's types, so it compiles against them unchanged
 * (Eigen::SparseMatrix<double, ColMajor, int> in compressed mode,
 * Eigen::MatrixXd, SymbolicFactor, DenseLDLTOptions, Inertia) and against
 * any stand-in with the same members:
 *
 *   SparseMatrixT  rows(), outerIndexPtr(), innerIndexPtr(), valuePtr()
 *   DenseMatrixT   DenseMatrixT(rows, cols), rows(), cols(), data() (column-major)
 *   SymbolicFactorT perm (data(), size()), etree.n, etree.parent (data()),
 *                  supernodes[i].firstCol / .ncols / .rowPattern (symbolic.hpp:138-199)
 *   OptionsT       zero_tolerance, relative_pivot_floor, pivot_threshold
 *                  (DenseLDLTOptions, dense_kernel.hpp:57-116)
 *   InertiaT       n_pos, n_neg, n_zero (inertia.hpp:14-18)
 *
 * Errors map onto the reference's exceptions (solver.hpp:141-143, :199-209,
 * :301-311, :403-413): std::logic_error, std::invalid_argument,
 * std::runtime_error, with symla_last_error() as the message.
 */
#ifndef SYMLA_GPU_BACKEND_HPP_
#define SYMLA_GPU_BACKEND_HPP_

#include <stdexcept>
#include <string>
#include <vector>

#include "symla_gpu.h"

namespace symla_gpu_backend {

inline void check(int rc) {
  if (rc == SYMLA_OK) return;
  const std::string msg = symla_last_error();
  if (rc == SYMLA_ERR_NOT_ANALYZED || rc == SYMLA_ERR_NOT_FACTORIZED || rc == SYMLA_ERR_SINGULAR)
    throw std::logic_error(msg);
  if (rc == SYMLA_ERR_BAD_SIZE || rc == SYMLA_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

class Backend {
 public:
  Backend() = default;
  Backend(const Backend&) = delete;
  Backend& operator=(const Backend&) = delete;
  ~Backend() { reset(); }

  void reset() {
    symla_gpu_destroy(ctx_);
    symla_symbolic_destroy(sym_);
    ctx_ = nullptr;
    sym_ = nullptr;
    factorized_ = false;
  }

  // SymLDLT::analyzePattern (solver.hpp:133-137): imports the SymbolicFactor
  // the reference computed (perm, etree parent, final supernodes) and builds
  // the device plan for A's pattern, which later factorizations reuse.
  template <class SymbolicFactorT, class SparseMatrixT>
  void analyze(const SymbolicFactorT& sf, const SparseMatrixT& A, int device = 0) {
    reset();
    std::vector<int> first, ncols, ptr{0}, rows;
    for (const auto& s : sf.supernodes) {
      first.push_back(s.firstCol);
      ncols.push_back(s.ncols);
      rows.insert(rows.end(), s.rowPattern.begin(), s.rowPattern.end());
      ptr.push_back(static_cast<int>(rows.size()));
    }
    const int n = static_cast<int>(sf.etree.n);
    check(symla_symbolic_import(n, sf.perm.data(), sf.etree.parent.data(), static_cast<int>(first.size()),
                                first.data(), ncols.data(), ptr.data(), rows.data(), &sym_));
    n_ = static_cast<int>(A.rows());
    check(symla_gpu_create(sym_, n_, A.outerIndexPtr(), A.innerIndexPtr(), device, &ctx_));
  }

  // SymLDLT::factorize, Mode::ThresholdPivot (solver.hpp:140-163), in place
  // of MultifrontalFactorizer<double>::factorize (multifrontal.hpp:299-300).
  template <class InertiaT, class SparseMatrixT, class OptionsT>
  InertiaT factorize(const SparseMatrixT& A, const OptionsT& o) {
    requireAnalyzed("symla::SymLDLT::factorize: analyzePattern must be called first");
    symla_factor_opts fo;
    symla_factor_opts_default(&fo);
    fo.mode = SYMLA_MODE_THRESHOLD;
    fo.pivot_threshold = o.pivot_threshold;
    fo.zero_tolerance = o.zero_tolerance;
    fo.relative_pivot_floor = o.relative_pivot_floor;
    return runFactorize<InertiaT>(A, fo);
  }

  // SymLDLT::factorizeStaticRegularized (solver.hpp:328-417) with
  // setKKTBlockSizes(n1, n2): the inertia-controlled delta retry loop.
  template <class InertiaT, class SparseMatrixT>
  InertiaT factorizeStaticRegularized(const SparseMatrixT& A, int n1, int n2, double initialDelta = 0.0,
                                      int maxRetries = 10, double growth = 10.0, double relFloor = 1e-8,
                                      double absFloor = 1e-300) {
    requireAnalyzed("symla::SymLDLT::factorize: analyzePattern must be called first");
    symla_regularize_opts ro;
    symla_regularize_opts_default(&ro);
    ro.initial_delta = initialDelta;
    ro.max_retries = maxRetries;
    ro.growth = growth;
    ro.static_rel_floor = relFloor;
    ro.static_abs_floor = absFloor;
    ro.kkt_n1 = n1;
    ro.kkt_n2 = n2;
    symla_factor_info info{};
    factorized_ = false;
    check(symla_gpu_factorize_regularized(ctx_, A.valuePtr(), 0, &ro, &info, &rinfo_));
    return finish<InertiaT>(info);
  }

  // SymLDLT::solve (solver.hpp:198-218), in place of
  // MultifrontalSolver<double>::solve (solve.hpp:159).
  template <class DenseMatrixT>
  DenseMatrixT solve(const DenseMatrixT& B) const {
    requireFactorized();
    if (static_cast<int>(B.rows()) != n_)
      throw std::invalid_argument("symla::SymLDLT::solve: B.rows() must match the factorized matrix size");
    DenseMatrixT X(B.rows(), B.cols());
    check(symla_gpu_solve(ctx_, B.data(), n_, static_cast<int>(B.cols()), X.data(), n_, 0));
    return X;
  }

  // SymLDLT::solveWithRefinement (solver.hpp:234-240): iterativeRefine
  // (refine.hpp:97-144) with the residual on the device.
  template <class SparseMatrixT, class DenseMatrixT>
  DenseMatrixT solveWithRefinement(const SparseMatrixT& A, const DenseMatrixT& B, int maxIterations = 10,
                                   double tolerance = 1e-14, symla_refine_info* info = nullptr) const {
    requireFactorized();
    if (static_cast<int>(B.rows()) != n_)
      throw std::invalid_argument("symla::SymLDLT::solve: B.rows() must match the factorized matrix size");
    DenseMatrixT X(B.rows(), B.cols());
    symla_refine_info ri{};
    check(symla_gpu_solve_refine(ctx_, A.valuePtr(), B.data(), n_, static_cast<int>(B.cols()), X.data(), n_, 0,
                                 maxIterations, tolerance, &ri));
    if (info) *info = ri;
    return X;
  }

  bool isSingular() const { return factorized_ && last_.singular != 0; }
  int regularizationRetriesUsed() const { return rinfo_.retries_used; }
  double lastRegularizationDelta() const { return rinfo_.last_delta; }
  const symla_factor_info& lastInfo() const { return last_; }
  symla_gpu_ctx* context() const { return ctx_; }

 private:
  void requireAnalyzed(const char* msg) const {
    if (!ctx_) throw std::logic_error(msg);
  }
  void requireFactorized() const {
    if (!factorized_) throw std::logic_error("symla::SymLDLT::solve: factorize() must be called before solve()");
  }
  template <class InertiaT, class SparseMatrixT>
  InertiaT runFactorize(const SparseMatrixT& A, const symla_factor_opts& fo) {
    symla_factor_info info{};
    factorized_ = false;
    check(symla_gpu_factorize(ctx_, A.valuePtr(), 0, &fo, &info));
    return finish<InertiaT>(info);
  }
  template <class InertiaT>
  InertiaT finish(const symla_factor_info& info) {
    last_ = info;
    factorized_ = true;
    InertiaT in{};
    in.n_pos = info.n_pos;
    in.n_neg = info.n_neg;
    in.n_zero = info.n_zero;
    return in;
  }

  symla_symbolic* sym_ = nullptr;
  symla_gpu_ctx* ctx_ = nullptr;
  int n_ = 0;
  bool factorized_ = false;
  symla_factor_info last_{};
  symla_regularize_info rinfo_{};
};

}  // namespace symla_gpu_backend

#endif  // SYMLA_GPU_BACKEND_HPP_
