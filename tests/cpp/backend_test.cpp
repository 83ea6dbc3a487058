// Drives include/symla_gpu_backend.hpp the way symla's SymLDLT<double> would
// (solver.hpp:133-240): analyzePattern -> import of a SymbolicFactor ->
// factorize -> solve -> solveWithRefinement, on the shifted 7-point
// Laplacian L7(k^3) - 2I with AMD ordering. The reference's Eigen containers
// and SymbolicFactor are replaced by minimal stand-ins with the same member
// names (Eigen is not installed here); the SymbolicFactor is filled from the
// library's own host analysis, as the reference's analyzePattern would fill
// its own. Exit 0 and one "backend_test OK" line on success.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "symla_gpu_backend.hpp"

namespace standin {
struct SparseMatrix {  // Eigen::SparseMatrix<double, ColMajor, int>, compressed
  int n = 0;
  std::vector<int> outer, inner;
  std::vector<double> values;
  int rows() const { return n; }
  const int* outerIndexPtr() const { return outer.data(); }
  const int* innerIndexPtr() const { return inner.data(); }
  const double* valuePtr() const { return values.data(); }
};
struct DenseMatrix {  // Eigen::MatrixXd (column-major)
  long r = 0, c = 0;
  std::vector<double> v;
  DenseMatrix(long rr, long cc) : r(rr), c(cc), v(static_cast<size_t>(rr * cc), 0.0) {}
  long rows() const { return r; }
  long cols() const { return c; }
  double* data() { return v.data(); }
  const double* data() const { return v.data(); }
};
struct Supernode {  // symbolic.hpp:138-159
  int firstCol = 0, ncols = 0;
  std::vector<int> rowPattern;
};
struct EliminationTree {  // elimination_tree.hpp:50-53
  std::vector<int> parent, colCount;
  int n = 0;
};
struct SymbolicFactor {  // symbolic.hpp:186-199
  std::vector<int> perm;
  EliminationTree etree;
  std::vector<Supernode> supernodes;
};
struct DenseLDLTOptions {  // dense_kernel.hpp:57-116
  double pivot_threshold = 0.01;
  double zero_tolerance = 1e-300;
  double relative_pivot_floor = 1e-12;
  int panel_size = 64;
};
struct Inertia {  // inertia.hpp:14-18
  int n_pos = 0, n_neg = 0, n_zero = 0;
};
}  // namespace standin

// Lower triangle of L7(k^3) - shift I (Dirichlet, centre 6, neighbours -1).
static standin::SparseMatrix laplacian7_lower(int k, double shift) {
  standin::SparseMatrix A;
  A.n = k * k * k;
  A.outer.push_back(0);
  for (int z = 0; z < k; ++z)
    for (int y = 0; y < k; ++y)
      for (int x = 0; x < k; ++x) {
        const int j = x + k * (y + k * z);
        A.inner.push_back(j);
        A.values.push_back(6.0 - shift);
        if (x + 1 < k) { A.inner.push_back(j + 1); A.values.push_back(-1.0); }
        if (y + 1 < k) { A.inner.push_back(j + k); A.values.push_back(-1.0); }
        if (z + 1 < k) { A.inner.push_back(j + k * k); A.values.push_back(-1.0); }
        A.outer.push_back(static_cast<int>(A.inner.size()));
      }
  return A;
}

// SymLDLT::analyzePattern's SymbolicFactor, here from the library's host
// analysis (symla_analyze + symla_symbolic_get).
static standin::SymbolicFactor analysis_of(const standin::SparseMatrix& A) {
  symla_symbolic* sym = nullptr;
  symla_gpu_backend::check(symla_analyze(A.n, A.outer.data(), A.inner.data(), SYMLA_ORDER_AMD, 64, 0.25, &sym));
  symla_symbolic_info info{};
  symla_gpu_backend::check(symla_symbolic_get_info(sym, &info));
  standin::SymbolicFactor sf;
  sf.perm.resize(info.n);
  sf.etree.n = info.n;
  sf.etree.parent.resize(info.n);
  sf.etree.colCount.resize(info.n);
  std::vector<int> first(info.num_supernodes), ncols(info.num_supernodes), ptr(info.num_supernodes + 1),
      rows(static_cast<size_t>(info.pattern_len));
  symla_gpu_backend::check(symla_symbolic_get(sym, sf.perm.data(), sf.etree.parent.data(), sf.etree.colCount.data(),
                                              first.data(), ncols.data(), ptr.data(), rows.data()));
  for (int s = 0; s < info.num_supernodes; ++s)
    sf.supernodes.push_back({first[s], ncols[s], std::vector<int>(rows.begin() + ptr[s], rows.begin() + ptr[s + 1])});
  symla_symbolic_destroy(sym);
  return sf;
}

// ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), A from its lower triangle.
static double backward_error(const standin::SparseMatrix& A, const standin::DenseMatrix& X,
                             const standin::DenseMatrix& B) {
  std::vector<double> r(B.v), rowsum(A.n, 0.0);
  for (int j = 0; j < A.n; ++j)
    for (int p = A.outer[j]; p < A.outer[j + 1]; ++p) {
      const int i = A.inner[p];
      const double a = A.values[p];
      r[i] -= a * X.v[j];
      rowsum[j] += std::fabs(a);
      if (i != j) r[j] -= a * X.v[i];
    }
  double rn = 0, an = 0, xn = 0, bn = 0;
  for (int i = 0; i < A.n; ++i) {
    rn = std::fmax(rn, std::fabs(r[i]));
    an = std::fmax(an, rowsum[i]);
    xn = std::fmax(xn, std::fabs(X.v[i]));
    bn = std::fmax(bn, std::fabs(B.v[i]));
  }
  return rn / (an * xn + bn);
}

int main(int argc, char** argv) {
  const int k = argc > 1 ? std::atoi(argv[1]) : 20;
  const standin::SparseMatrix A = laplacian7_lower(k, 2.0);
  const standin::SymbolicFactor sf = analysis_of(A);
  symla_gpu_backend::Backend gpu;
  bool threw = false;
  try {
    standin::DenseLDLTOptions o;
    gpu.factorize<standin::Inertia>(A, o);
  } catch (const std::logic_error&) {
    threw = true;  // factorize before analyzePattern (solver.hpp:141-143)
  }
  if (!threw) { std::printf("backend_test FAIL: no logic_error before analyze\n"); return 1; }
  gpu.analyze(sf, A);
  const standin::Inertia in = gpu.factorize<standin::Inertia>(A, standin::DenseLDLTOptions{});
  standin::DenseMatrix B(A.n, 1);
  for (int i = 0; i < A.n; ++i) B.v[i] = 1.0 + 0.001 * (i % 7);
  const standin::DenseMatrix X = gpu.solve(B);
  const double e0 = backward_error(A, X, B);
  symla_refine_info ri{};
  const standin::DenseMatrix Xr = gpu.solveWithRefinement(A, B, 10, 1e-12, &ri);
  const double e1 = backward_error(A, Xr, B);
  threw = false;
  try {
    gpu.solve(standin::DenseMatrix(A.n + 1, 1));
  } catch (const std::invalid_argument&) {
    threw = true;  // B.rows() mismatch (solver.hpp:207-209)
  }
  std::printf("backend_test n=%d inertia=(%d,%d,%d) backward_error=%.3e refined=%.3e size_error_thrown=%d\n", A.n,
              in.n_pos, in.n_neg, in.n_zero, e0, e1, threw ? 1 : 0);
  const bool ok = threw && e0 < 1e-10 && e1 <= 1e-12 && in.n_pos + in.n_neg + in.n_zero == A.n &&
                  (k != 20 || (in.n_pos == 7590 && in.n_neg == 410 && in.n_zero == 0));
  std::printf(ok ? "backend_test OK\n" : "backend_test FAIL\n");
  return ok ? 0 : 1;
}
