// ORACLE -- test infrastructure only (see oracle.hpp).
// Flat C interface over the oracle, loaded by tests/ and bench.py through
// ctypes. Error codes: 0 ok, 1 std::logic_error, 2 std::invalid_argument,
// 3 std::runtime_error, 4 other exception.
#include <cstring>
#include <stdexcept>
#include <string>

#include "oracle.hpp"

using namespace oracle;

namespace {
int fail(char* err, int errlen, int code, const char* what) {
  if (err && errlen > 0) {
    std::strncpy(err, what, errlen - 1);
    err[errlen - 1] = 0;
  }
  return code;
}
template <typename F>
int guarded(char* err, int errlen, F&& body) {
  try {
    body();
  } catch (const std::invalid_argument& e) {
    return fail(err, errlen, 2, e.what());
  } catch (const std::logic_error& e) {
    return fail(err, errlen, 1, e.what());
  } catch (const std::runtime_error& e) {
    return fail(err, errlen, 3, e.what());
  } catch (const std::exception& e) {
    return fail(err, errlen, 4, e.what());
  }
  return 0;
}
}  // namespace

extern "C" {

void* oracle_solver_create(int n, const int* perm, const int* parent, int numSN, const int* snFirst,
                           const int* snNcols, const int* snPtr, const int* snRows) {
  auto* s = new SymLDLT();
  Symbolic sym;
  sym.n = n;
  sym.perm.assign(perm, perm + n);
  sym.parent.assign(parent, parent + n);
  sym.supernodes.resize(numSN);
  for (int i = 0; i < numSN; ++i) {
    sym.supernodes[i].firstCol = snFirst[i];
    sym.supernodes[i].ncols = snNcols[i];
    sym.supernodes[i].rowPattern.assign(snRows + snPtr[i], snRows + snPtr[i + 1]);
  }
  s->setSymbolic(std::move(sym));
  return s;
}

void oracle_solver_destroy(void* h) { delete static_cast<SymLDLT*>(h); }

int oracle_set(void* h, const char* name, double value) {
  auto* s = static_cast<SymLDLT*>(h);
  const std::string k(name);
  if (k == "mode")
    s->mode = value > 0.5 ? Mode::StaticRegularized : Mode::ThresholdPivot;
  else if (k == "parallel")
    s->parallel = value != 0.0;
  else if (k == "num_threads")
    s->num_threads = static_cast<int>(value);
  else if (k == "pivot_threshold")
    s->pivot_threshold = value;
  else if (k == "zero_tolerance")
    s->zero_tolerance = value;
  else if (k == "relative_pivot_floor")
    s->relative_pivot_floor = value;
  else if (k == "initial_delta")
    s->initial_regularization_delta = value;
  else if (k == "max_retries")
    s->max_regularization_retries = static_cast<int>(value);
  else if (k == "growth")
    s->regularization_growth = value;
  else if (k == "static_rel_floor")
    s->static_pivot_relative_floor = value;
  else if (k == "static_abs_floor")
    s->static_pivot_absolute_floor = value;
  else
    return -1;
  return 0;
}

int oracle_set_kkt(void* h, int n1, int n2) {
  auto* s = static_cast<SymLDLT*>(h);
  if (n1 < 0 || n2 < 0) return 2;
  s->kkt_n1 = n1;
  s->kkt_n2 = n2;
  s->use_kkt_blocks = true;
  s->use_explicit_signs = false;
  return 0;
}

int oracle_set_signs(void* h, int n, const int* signs) {
  auto* s = static_cast<SymLDLT*>(h);
  s->expected_signs_orig.assign(signs, signs + n);
  s->use_explicit_signs = true;
  s->use_kkt_blocks = false;
  return 0;
}

int oracle_factorize(void* h, int n, const int* colptr, const int* rowind, const double* vals, char* err, int errlen) {
  auto* s = static_cast<SymLDLT*>(h);
  return guarded(err, errlen, [&] {
    Csc A{n, colptr, rowind, vals};
    s->factorize(A);
  });
}

// ints: n_pos, n_neg, n_zero, singular, n_singular, retries, num_perturbed,
//       num_delayed, factorized, num_fronts
// dbls: last_delta, total_perturbation
void oracle_info(void* h, int* ints, double* dbls) {
  auto* s = static_cast<SymLDLT*>(h);
  const auto& nf = s->numeric;
  ints[0] = nf.inertia.n_pos;
  ints[1] = nf.inertia.n_neg;
  ints[2] = nf.inertia.n_zero;
  ints[3] = nf.singular ? 1 : 0;
  ints[4] = static_cast<int>(nf.singularCols.size());
  ints[5] = s->regularization_retries_used;
  ints[6] = nf.numPerturbed;
  ints[7] = nf.numDelayedColumns;
  ints[8] = s->factorized ? 1 : 0;
  ints[9] = static_cast<int>(nf.fronts.size());
  dbls[0] = s->last_regularization_delta;
  dbls[1] = nf.totalPerturbation;
}

int oracle_singular_cols(void* h, int* out) {
  auto* s = static_cast<SymLDLT*>(h);
  const auto& c = s->numeric.singularCols;
  for (size_t i = 0; i < c.size(); ++i) out[i] = c[i];
  return static_cast<int>(c.size());
}

int oracle_attempts(void* h, double* deltas, int* ok, int cap) {
  auto* s = static_cast<SymLDLT*>(h);
  const int k = static_cast<int>(s->attemptDeltas.size());
  for (int i = 0; i < k && i < cap; ++i) {
    deltas[i] = s->attemptDeltas[i];
    ok[i] = s->attemptOk[i];
  }
  return k;
}

int oracle_solve(void* h, const double* B, int n, int nrhs, double* X, char* err, int errlen) {
  auto* s = static_cast<SymLDLT*>(h);
  return guarded(err, errlen, [&] {
    Mat Bm(n, nrhs);
    std::memcpy(Bm.a.data(), B, sizeof(double) * static_cast<size_t>(n) * nrhs);
    Mat Xm = s->solve(Bm);
    std::memcpy(X, Xm.a.data(), sizeof(double) * static_cast<size_t>(n) * nrhs);
  });
}

int oracle_refine(void* h, int n, const int* colptr, const int* rowind, const double* vals, const double* B, int nrhs,
                  double* X, int maxIt, double tol, int* iters, double* initRes, double* finalRes, char* err,
                  int errlen) {
  auto* s = static_cast<SymLDLT*>(h);
  return guarded(err, errlen, [&] {
    Csc A{n, colptr, rowind, vals};
    Mat Bm(n, nrhs);
    std::memcpy(Bm.a.data(), B, sizeof(double) * static_cast<size_t>(n) * nrhs);
    Mat Xm;
    RefinementOptions o;
    o.max_iterations = maxIt;
    o.tolerance = tol;
    RefinementResult r = s->solveWithRefinement(A, Bm, Xm, o);
    std::memcpy(X, Xm.a.data(), sizeof(double) * static_cast<size_t>(n) * nrhs);
    *iters = r.iterations;
    *initRes = r.initial_relative_residual;
    *finalRes = r.final_relative_residual;
  });
}

// Per-front sizes: m[si] = rowIndices.size(), npiv[si] = nPivots.
void oracle_front_sizes(void* h, int* m, int* npiv) {
  auto* s = static_cast<SymLDLT*>(h);
  const auto& fr = s->numeric.fronts;
  for (size_t i = 0; i < fr.size(); ++i) {
    m[i] = static_cast<int>(fr[i].rowIndices.size());
    npiv[i] = fr[i].nPivots;
  }
}

// Front si: rowIndices (m), L (m x npiv column-major), D diag/offdiag (npiv),
// pivot blocks (start, kind) -> returns the number of pivot blocks.
int oracle_front_get(void* h, int si, int* rowIndices, double* L, double* Ddiag, double* Doff, int* pivStart,
                     int* pivKind) {
  auto* s = static_cast<SymLDLT*>(h);
  const auto& f = s->numeric.fronts[si];
  const int m = static_cast<int>(f.rowIndices.size());
  for (int i = 0; i < m; ++i) rowIndices[i] = f.rowIndices[i];
  std::memcpy(L, f.L.a.data(), sizeof(double) * f.L.a.size());
  for (int i = 0; i < f.nPivots; ++i) {
    Ddiag[i] = f.D.diag[i];
    Doff[i] = f.D.offdiag[i];
  }
  for (size_t b = 0; b < f.pivotBlocks.size(); ++b) {
    pivStart[b] = f.pivotBlocks[b].start;
    pivKind[b] = static_cast<int>(f.pivotBlocks[b].kind);
  }
  return static_cast<int>(f.pivotBlocks.size());
}

// Dense kernel on an n x n column-major matrix (lower triangle read), in
// place. isStatic selects factorStatic. ints out: n_factored, n_pos, n_neg,
// n_zero, num_pivot_blocks, num_perturbed. dbl out: max_growth,
// total_perturbation.
int oracle_dense_factor(int n, double* A, int lda, int nEligible, int isStatic, double zeroTol, double relFloor,
                        int panelSize, double delta, double staticRelFloor, double staticAbsFloor,
                        const int* expectedSign, int nSign, int* perm, double* Ddiag, double* Doff, int* pivStart,
                        int* pivKind, int* ints, double* dbls, char* err, int errlen) {
  return guarded(err, errlen, [&] {
    MatView V{A, n, n, lda};
    BlockDiagonalD D;
    DenseLDLTResult r;
    if (isStatic) {
      StaticPivotOptions o;
      o.delta = delta;
      o.relative_pivot_floor = staticRelFloor;
      o.absolute_floor = staticAbsFloor;
      o.panel_size = panelSize;
      std::vector<int> sg(expectedSign, expectedSign + nSign);
      r = denseFactorStatic(V, D, o, sg, nEligible);
    } else {
      DenseLDLTOptions o;
      o.zero_tolerance = zeroTol;
      o.relative_pivot_floor = relFloor;
      o.panel_size = panelSize;
      r = denseFactor(V, D, o, nEligible);
    }
    for (int i = 0; i < n; ++i) {
      perm[i] = r.perm[i];
      Ddiag[i] = D.diag[i];
      Doff[i] = D.offdiag[i];
    }
    for (size_t b = 0; b < r.pivots.size(); ++b) {
      pivStart[b] = r.pivots[b].start;
      pivKind[b] = static_cast<int>(r.pivots[b].kind);
    }
    ints[0] = r.n_factored;
    ints[1] = r.inertia.n_pos;
    ints[2] = r.inertia.n_neg;
    ints[3] = r.inertia.n_zero;
    ints[4] = static_cast<int>(r.pivots.size());
    ints[5] = r.num_perturbed;
    dbls[0] = r.max_growth;
    dbls[1] = r.total_perturbation;
  });
}

}  // extern "C"
