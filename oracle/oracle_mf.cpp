// ORACLE -- test infrastructure only (see oracle.hpp).
// Restatement of include/symla/multifrontal.hpp, solve.hpp, refine.hpp,
// solver.hpp and parallel/task_graph.hpp.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <limits>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.hpp"

namespace oracle {

namespace {

// parallel/task_graph.hpp:48-89
template <typename ProcessFn>
void runTaskDag(const std::vector<int>& roots, const std::vector<std::vector<int>>& children,
                const std::vector<long long>& subtreeWeight, long long taskCutoff, ProcessFn&& process) {
#ifdef _OPENMP
  std::function<void(int)> visit = [&](int node) {
    bool spawnedAny = false;
    for (int c : children[node]) {
      if (subtreeWeight[c] >= taskCutoff) {
        spawnedAny = true;
#pragma omp task default(shared) firstprivate(c)
        visit(c);
      } else {
        visit(c);
      }
    }
    if (spawnedAny) {
#pragma omp taskwait
    }
    process(node);
  };
  for (int r : roots) {
#pragma omp task default(shared) firstprivate(r)
    visit(r);
  }
#pragma omp taskwait
#else
  std::function<void(int)> visit = [&](int node) {
    for (int c : children[node]) visit(c);
    process(node);
  };
  for (int r : roots) visit(r);
#endif
}

// parallel/task_graph.hpp:108-153
template <typename ProcessFn>
void runTaskDagTopDown(const std::vector<int>& roots, const std::vector<std::vector<int>>& children,
                       const std::vector<long long>& subtreeWeight, long long taskCutoff, ProcessFn&& process) {
#ifdef _OPENMP
  std::function<void(int)> visit = [&](int node) {
    process(node);
    for (int c : children[node]) {
      if (subtreeWeight[c] >= taskCutoff) {
#pragma omp task default(shared) firstprivate(c)
        visit(c);
      } else {
        visit(c);
      }
    }
  };
#pragma omp taskgroup
  {
    for (int r : roots) {
#pragma omp task default(shared) firstprivate(r)
      visit(r);
    }
  }
#else
  std::function<void(int)> visit = [&](int node) {
    process(node);
    for (int c : children[node]) visit(c);
  };
  for (int r : roots) visit(r);
#endif
}

int maxThreadsFor(bool parallel, int num_threads) {
#ifdef _OPENMP
  return parallel ? std::max(1, num_threads > 0 ? num_threads : omp_get_max_threads()) : 1;
#else
  (void)parallel;
  (void)num_threads;
  return 1;
#endif
}

int threadId(bool parallel) {
#ifdef _OPENMP
  return parallel ? omp_get_thread_num() : 0;
#else
  (void)parallel;
  return 0;
#endif
}

// multifrontal.hpp:199-242 -- lower triangle of A in final order, rows sorted.
struct PermutedLower {
  std::vector<std::vector<int>> rows;
  std::vector<std::vector<double>> vals;
  static PermutedLower build(const Csc& A, const std::vector<int>& perm) {
    const int n = A.n;
    std::vector<int> newIndexOf(n);
    for (int k = 0; k < n; ++k) newIndexOf[perm[k]] = k;
    PermutedLower out;
    out.rows.resize(n);
    out.vals.resize(n);
    for (int c = 0; c < n; ++c) {
      for (int p = A.colptr[c]; p < A.colptr[c + 1]; ++p) {
        const int r = A.rowind[p];
        if (r < c) continue;
        const int nr = newIndexOf[r], nc = newIndexOf[c];
        const int lo = std::min(nr, nc), hi = std::max(nr, nc);
        out.rows[lo].push_back(hi);
        out.vals[lo].push_back(A.vals[p]);
      }
    }
    for (int c = 0; c < n; ++c) {
      std::vector<int> order(out.rows[c].size());
      for (size_t k = 0; k < order.size(); ++k) order[k] = static_cast<int>(k);
      std::sort(order.begin(), order.end(), [&](int a, int b) { return out.rows[c][a] < out.rows[c][b]; });
      std::vector<int> nr(order.size());
      std::vector<double> nv(order.size());
      for (size_t k = 0; k < order.size(); ++k) {
        nr[k] = out.rows[c][order[k]];
        nv[k] = out.vals[c][order[k]];
      }
      out.rows[c].swap(nr);
      out.vals[c].swap(nv);
    }
    return out;
  }
};

}  // namespace

NumericFactor multifrontalFactorize(const Symbolic& sf, const Csc& A, const DenseLDLTOptions& options,
                                    const MultifrontalOptions& mfOptions) {
  const int n = sf.n;
  NumericFactor nf;
  nf.perm = sf.perm;
  nf.n = n;
  if (n == 0) return nf;
  const auto& supernodes = sf.supernodes;
  const int numSN = static_cast<int>(supernodes.size());

  // multifrontal.hpp:312-339
  std::vector<int> colToSupernode(n, -1);
  for (int si = 0; si < numSN; ++si)
    for (int c = supernodes[si].firstCol; c < supernodes[si].firstCol + supernodes[si].ncols; ++c)
      colToSupernode[c] = si;
  std::vector<int> parentSN(numSN, -1);
  std::vector<std::vector<int>> childrenSN(numSN);
  std::vector<int> rootsSN;
  for (int si = 0; si < numSN; ++si) {
    const int lastCol = supernodes[si].firstCol + supernodes[si].ncols - 1;
    const int p = sf.parent[lastCol];
    if (p != -1) {
      const int psn = colToSupernode[p];
      parentSN[si] = psn;
      childrenSN[psn].push_back(si);
    }
  }
  for (int si = 0; si < numSN; ++si)
    if (parentSN[si] == -1) rootsSN.push_back(si);
  nf.parentSN = parentSN;
  nf.childrenSN = childrenSN;
  nf.rootsSN = rootsSN;

  auto Aperm = PermutedLower::build(A, sf.perm);

  struct GeneratedElement {
    std::vector<int> indices;
    Mat matrix;
  };
  std::vector<GeneratedElement> genElem(numSN);
  nf.fronts.resize(numSN);
  std::vector<Inertia> perFrontInertia(numSN);
  std::vector<double> perFrontPerturbation(numSN, 0.0);
  std::vector<int> perFrontNumPerturbed(numSN, 0);
  std::vector<int> perFrontExtras(numSN, 0);
  std::mutex singularMutex;

  const int maxThreads = maxThreadsFor(mfOptions.parallel, mfOptions.num_threads);
  std::vector<std::vector<int>> globalToLocalTls(maxThreads, std::vector<int>(n, -1));

  // multifrontal.hpp:418-429
  std::vector<long long> subtreeWeight(numSN, 0);
  for (int si = 0; si < numSN; ++si) {
    const long long m = static_cast<long long>(supernodes[si].rowPattern.size());
    const long long snCols = supernodes[si].ncols;
    subtreeWeight[si] += std::max<long long>(1, snCols * m * m);
    const int p = parentSN[si];
    if (p != -1) subtreeWeight[p] += subtreeWeight[si];
  }
  long long totalCost = 0;
  for (int r : rootsSN) totalCost += subtreeWeight[r];

  // multifrontal.hpp:436-644
  auto processSupernode = [&](int si) {
    std::vector<int>& globalToLocal = globalToLocalTls[threadId(mfOptions.parallel)];
    const auto& sn = supernodes[si];
    const int ncols = sn.ncols;

    std::vector<int> extraFromChildren;
    for (int ci : childrenSN[si]) {
      for (int idx : genElem[ci].indices)
        if (!std::binary_search(sn.rowPattern.begin(), sn.rowPattern.end(), idx)) extraFromChildren.push_back(idx);
    }
    std::sort(extraFromChildren.begin(), extraFromChildren.end());
    extraFromChildren.erase(std::unique(extraFromChildren.begin(), extraFromChildren.end()),
                            extraFromChildren.end());
    const int nExtra = static_cast<int>(extraFromChildren.size());
    const int nEligible = ncols + nExtra;
    const int m = static_cast<int>(sn.rowPattern.size()) + nExtra;
    perFrontExtras[si] = nExtra;

    std::vector<int> frontIdx(m);
    for (int j = 0; j < ncols; ++j) frontIdx[j] = sn.firstCol + j;
    for (int j = 0; j < nExtra; ++j) frontIdx[ncols + j] = extraFromChildren[j];
    for (int j = ncols; j < static_cast<int>(sn.rowPattern.size()); ++j) frontIdx[nEligible + (j - ncols)] = sn.rowPattern[j];
    for (int t = 0; t < m; ++t) globalToLocal[frontIdx[t]] = t;

    Mat F(m, m);
    for (int j = 0; j < ncols; ++j) {
      const int gj = sn.firstCol + j;
      const auto& rr = Aperm.rows[gj];
      const auto& vv = Aperm.vals[gj];
      for (size_t t = 0; t < rr.size(); ++t) F(globalToLocal[rr[t]], j) += vv[t];
    }
    for (int ci : childrenSN[si]) {
      auto& ge = genElem[ci];
      const int p = static_cast<int>(ge.indices.size());
      for (int a = 0; a < p; ++a) {
        const int la = globalToLocal[ge.indices[a]];
        for (int b = 0; b <= a; ++b) {
          const int lb = globalToLocal[ge.indices[b]];
          const double v = ge.matrix(a, b);
          if (la >= lb)
            F(la, lb) += v;
          else
            F(lb, la) += v;
        }
      }
      ge.matrix = Mat();
      std::vector<int>().swap(ge.indices);
    }
    for (int t = 0; t < m; ++t) globalToLocal[frontIdx[t]] = -1;

    static constexpr int kPanelBlockingMinFront = 256;
    BlockDiagonalD D;
    DenseLDLTResult res;
    if (mfOptions.static_pivoting) {
      std::vector<int> localExpectedSign(m, 0);
      if (!mfOptions.expectedSign.empty()) {
        for (int t = 0; t < m; ++t) {
          const int g = frontIdx[t];
          if (g >= 0 && g < static_cast<int>(mfOptions.expectedSign.size())) localExpectedSign[t] = mfOptions.expectedSign[g];
        }
      }
      StaticPivotOptions so = mfOptions.staticOptions;
      if (nEligible < kPanelBlockingMinFront) so.panel_size = 1;
      res = denseFactorStatic(F.view(), D, so, localExpectedSign, nEligible);
    } else {
      DenseLDLTOptions fo = options;
      if (nEligible < kPanelBlockingMinFront) fo.panel_size = 1;
      res = denseFactor(F.view(), D, fo, nEligible);
    }
    perFrontInertia[si] = res.inertia;
    perFrontPerturbation[si] = res.total_perturbation;
    perFrontNumPerturbed[si] = res.num_perturbed;
    const int nFactored = res.n_factored;
    auto globalOf = [&](int i) { return frontIdx[res.perm[i]]; };

    SupernodeFactor sfac;
    sfac.nPivots = nFactored;
    sfac.rowIndices.resize(m);
    for (int i = 0; i < m; ++i) sfac.rowIndices[i] = globalOf(i);
    sfac.L = Mat(m, nFactored);
    for (int j = 0; j < nFactored; ++j)
      for (int i = 0; i < m; ++i) sfac.L(i, j) = F(i, j);
    sfac.D.diag.assign(D.diag.begin(), D.diag.begin() + nFactored);
    sfac.D.offdiag.assign(D.offdiag.begin(), D.offdiag.begin() + nFactored);
    sfac.pivotBlocks = res.pivots;
    sfac.Ltop = Mat(nFactored, nFactored);
    for (int j = 0; j < nFactored; ++j)
      for (int i = 0; i < nFactored; ++i) sfac.Ltop(i, j) = F(i, j);
    for (const auto& pb : sfac.pivotBlocks)
      if (pb.kind == PivotKind::TwoByTwo) sfac.Ltop(pb.start + 1, pb.start) = 0.0;
    nf.fronts[si] = std::move(sfac);

    const int leftover = m - nFactored;
    if (leftover > 0) {
      const int psn = parentSN[si];
      if (psn == -1) {
        std::lock_guard<std::mutex> lock(singularMutex);
        nf.singular = true;
        for (int i = nFactored; i < m; ++i) nf.singularCols.push_back(globalOf(i));
      } else {
        GeneratedElement ge;
        ge.indices.resize(leftover);
        for (int i = 0; i < leftover; ++i) ge.indices[i] = globalOf(nFactored + i);
        ge.matrix = Mat(leftover, leftover);
        for (int j = 0; j < leftover; ++j)
          for (int i = 0; i < leftover; ++i) ge.matrix(i, j) = F(nFactored + i, nFactored + j);
        genElem[si] = std::move(ge);
      }
    }
  };

#ifdef _OPENMP
  if (mfOptions.parallel) {
    // multifrontal.hpp:676-787
    int effectiveThreads = maxThreads;
    if (mfOptions.num_threads <= 0) {
      constexpr long long kCostPerThread = 8'000'000;
      const long long threadsFromCost = totalCost / kCostPerThread;
      effectiveThreads = static_cast<int>(std::min<long long>(maxThreads, std::max<long long>(1, threadsFromCost)));
    }
    long long cutoff = mfOptions.task_cutoff;
    if (cutoff < 0) {
      constexpr long long kTargetTasksPerThread = 4;
      const long long targetTasks = std::max<long long>(1, kTargetTasksPerThread * effectiveThreads);
      cutoff = totalCost > 0 ? std::max<long long>(1, totalCost / targetTasks) : 1;
      constexpr long long kMinTaskCost = 1 << 17;
      cutoff = std::max(cutoff, kMinTaskCost);
    }
    constexpr long long kMinTotalCostForParallel = (1 << 17) * 4;
    if (totalCost < kMinTotalCostForParallel) {
      for (int si = 0; si < numSN; ++si) processSupernode(si);
    } else {
      const int savedMaxActiveLevels = omp_get_max_active_levels();
      omp_set_max_active_levels(1);
      const int requestedThreads = mfOptions.num_threads > 0 ? mfOptions.num_threads : effectiveThreads;
#pragma omp parallel num_threads(requestedThreads)
      {
#pragma omp single
        { runTaskDag(rootsSN, childrenSN, subtreeWeight, cutoff, processSupernode); }
      }
      omp_set_max_active_levels(savedMaxActiveLevels);
    }
  } else {
    for (int si = 0; si < numSN; ++si) processSupernode(si);
  }
#else
  for (int si = 0; si < numSN; ++si) processSupernode(si);
#endif

  for (int si = 0; si < numSN; ++si) {
    nf.inertia.n_pos += perFrontInertia[si].n_pos;
    nf.inertia.n_neg += perFrontInertia[si].n_neg;
    nf.inertia.n_zero += perFrontInertia[si].n_zero;
    nf.totalPerturbation += perFrontPerturbation[si];
    nf.numPerturbed += perFrontNumPerturbed[si];
    nf.numDelayedColumns += perFrontExtras[si];
  }
  std::sort(nf.singularCols.begin(), nf.singularCols.end());
  return nf;
}

// ---------------------------------------------------------------------------
// solve.hpp
namespace {

// Unit-lower triangular solve Ltop * Y = Y (in place), k x nrhs, Y ld = k.
void unitLowerSolve(const Mat& Ltop, double* Y, int k, int nrhs) {
  for (int c = 0; c < nrhs; ++c) {
    double* y = Y + static_cast<size_t>(c) * k;
    for (int j = 0; j < k; ++j) {
      const double yj = y[j];
      if (yj == 0.0) continue;
      for (int i = j + 1; i < k; ++i) y[i] -= Ltop(i, j) * yj;
    }
  }
}
// Ltop^T * X = X (unit upper), in place.
void unitLowerTransSolve(const Mat& Ltop, double* X, int k, int nrhs) {
  for (int c = 0; c < nrhs; ++c) {
    double* x = X + static_cast<size_t>(c) * k;
    for (int j = k - 1; j >= 0; --j) {
      double s = x[j];
      for (int i = j + 1; i < k; ++i) s -= Ltop(i, j) * x[i];
      x[j] = s;
    }
  }
}

void diagonalSolve(const NumericFactor& nf, const Mat& Y, Mat& Z) {
  const int nrhs = Y.cols;
  for (const auto& f : nf.fronts) {
    for (const auto& pb : f.pivotBlocks) {
      const int s = pb.start;
      if (pb.kind == PivotKind::OneByOne) {
        const int idx = f.rowIndices[s];
        for (int c = 0; c < nrhs; ++c) Z(idx, c) = Y(idx, c) / f.D.diag[s];
      } else {
        const int i0 = f.rowIndices[s], i1 = f.rowIndices[s + 1];
        const double d11 = f.D.diag[s], d21 = f.D.offdiag[s], d22 = f.D.diag[s + 1];
        const double det = d11 * d22 - d21 * d21;
        for (int c = 0; c < nrhs; ++c) {
          const double y0 = Y(i0, c), y1 = Y(i1, c);
          Z(i0, c) = (d22 * y0 - d21 * y1) / det;
          Z(i1, c) = (-d21 * y0 + d11 * y1) / det;
        }
      }
    }
  }
}

}  // namespace

Mat multifrontalSolve(const NumericFactor& nf, const Mat& B, const SolveOptions& so) {
  const int n = nf.n;
  if (B.rows != n) throw std::invalid_argument("symla::MultifrontalSolver::solve: B.rows() must match the factorized matrix size");
  const int nrhs = B.cols;
  if (n == 0) return Mat(0, nrhs);
  Mat Bp(n, nrhs);
  for (int t = 0; t < n; ++t)
    for (int c = 0; c < nrhs; ++c) Bp(t, c) = B(nf.perm[t], c);
  const int numSN = static_cast<int>(nf.fronts.size());

  const int maxThreads = maxThreadsFor(so.parallel, so.num_threads);
  std::vector<long long> subtreeWeight(numSN, 0);
  for (int si = 0; si < numSN; ++si) {
    const auto& f = nf.fronts[si];
    const long long m = static_cast<long long>(f.rowIndices.size());
    const long long k = std::max<long long>(1, f.nPivots);
    subtreeWeight[si] += std::max<long long>(1, m * k) * std::max(1, nrhs);
    const int p = nf.parentSN[si];
    if (p != -1) subtreeWeight[p] += subtreeWeight[si];
  }
  long long totalCost = 0;
  for (int r : nf.rootsSN) totalCost += subtreeWeight[r];

  bool runParallel = false;
  long long cutoff = 0;
  int requestedThreads = 1;
#ifdef _OPENMP
  if (so.parallel && numSN > 0) {
    constexpr long long kCostPerThread = 2'000'000;
    int effectiveThreads = maxThreads;
    if (so.num_threads <= 0) {
      const long long threadsFromCost = totalCost / kCostPerThread;
      effectiveThreads = static_cast<int>(std::min<long long>(maxThreads, std::max<long long>(1, threadsFromCost)));
    }
    cutoff = so.task_cutoff;
    if (cutoff < 0) {
      constexpr long long kTargetTasksPerThread = 4;
      const long long targetTasks = std::max<long long>(1, kTargetTasksPerThread * effectiveThreads);
      cutoff = totalCost > 0 ? std::max<long long>(1, totalCost / targetTasks) : 1;
      constexpr long long kMinTaskCost = 1'000'000;
      cutoff = std::max(cutoff, kMinTaskCost);
    }
    long long maxSpawnable = 0;
    for (int si = 0; si < numSN; ++si)
      if (nf.parentSN[si] != -1) maxSpawnable = std::max(maxSpawnable, subtreeWeight[si]);
    if (nf.rootsSN.size() >= 2)
      for (int r : nf.rootsSN) maxSpawnable = std::max(maxSpawnable, subtreeWeight[r]);
    constexpr long long kMinTotalCostForParallel = 1'000'000 * 4;
    if ((totalCost >= kMinTotalCostForParallel && maxSpawnable >= cutoff) || so.task_cutoff >= 0) {
      runParallel = true;
      requestedThreads = so.num_threads > 0 ? so.num_threads : effectiveThreads;
    }
  }
#endif
  (void)maxThreads;

  Mat Y(n, nrhs), Z(n, nrhs), X(n, nrhs);
  if (runParallel) {
#ifdef _OPENMP
    struct RhsElement {
      std::vector<int> indices;
      Mat matrix;
    };
    std::vector<RhsElement> rhsElem(numSN);
    std::vector<std::vector<int>> globalToLocalTls(std::max(1, requestedThreads), std::vector<int>(n, -1));
    auto forwardProcess = [&](int si) {
      std::vector<int>& g2l = globalToLocalTls[omp_get_thread_num()];
      const auto& f = nf.fronts[si];
      const int m = static_cast<int>(f.rowIndices.size());
      const int k = f.nPivots;
      if (m == 0) return;
      Mat G(m, nrhs);
      for (int t = 0; t < m; ++t) g2l[f.rowIndices[t]] = t;
      for (int ci : nf.childrenSN[si]) {
        RhsElement& ce = rhsElem[ci];
        const int p = static_cast<int>(ce.indices.size());
        for (int a = 0; a < p; ++a) {
          const int li = g2l[ce.indices[a]];
          for (int c = 0; c < nrhs; ++c) G(li, c) += ce.matrix(a, c);
        }
        ce.matrix = Mat();
        std::vector<int>().swap(ce.indices);
      }
      for (int t = 0; t < m; ++t) g2l[f.rowIndices[t]] = -1;
      std::vector<double> yOwn(static_cast<size_t>(k) * nrhs);
      if (k > 0) {
        for (int p = 0; p < k; ++p)
          for (int c = 0; c < nrhs; ++c) yOwn[p + static_cast<size_t>(c) * k] = Bp(f.rowIndices[p], c) - G(p, c);
        unitLowerSolve(f.Ltop, yOwn.data(), k, nrhs);
        for (int p = 0; p < k; ++p)
          for (int c = 0; c < nrhs; ++c) Y(f.rowIndices[p], c) = yOwn[p + static_cast<size_t>(c) * k];
      }
      const int extra = m - k;
      if (extra > 0) {
        Mat newExtra(extra, nrhs);
        for (int c = 0; c < nrhs; ++c)
          for (int i = 0; i < extra; ++i) newExtra(i, c) = G(k + i, c);
        if (k > 0) {
          for (int c = 0; c < nrhs; ++c)
            for (int p = 0; p < k; ++p) {
              const double yv = yOwn[p + static_cast<size_t>(c) * k];
              for (int i = 0; i < extra; ++i) newExtra(i, c) += f.L(k + i, p) * yv;
            }
        }
        rhsElem[si].indices.assign(f.rowIndices.begin() + k, f.rowIndices.end());
        rhsElem[si].matrix = std::move(newExtra);
      }
    };
    auto backwardProcess = [&](int si) {
      const auto& f = nf.fronts[si];
      const int m = static_cast<int>(f.rowIndices.size());
      const int k = f.nPivots;
      if (k == 0) return;
      std::vector<double> xOwn(static_cast<size_t>(k) * nrhs);
      for (int p = 0; p < k; ++p)
        for (int c = 0; c < nrhs; ++c) xOwn[p + static_cast<size_t>(c) * k] = Z(f.rowIndices[p], c);
      const int extra = m - k;
      if (extra > 0) {
        for (int c = 0; c < nrhs; ++c)
          for (int p = 0; p < k; ++p) {
            double s = 0.0;
            for (int i = 0; i < extra; ++i) s += f.L(k + i, p) * X(f.rowIndices[k + i], c);
            xOwn[p + static_cast<size_t>(c) * k] -= s;
          }
      }
      unitLowerTransSolve(f.Ltop, xOwn.data(), k, nrhs);
      for (int p = 0; p < k; ++p)
        for (int c = 0; c < nrhs; ++c) X(f.rowIndices[p], c) = xOwn[p + static_cast<size_t>(c) * k];
    };
    const int savedMaxActiveLevels = omp_get_max_active_levels();
    omp_set_max_active_levels(1);
#pragma omp parallel num_threads(requestedThreads)
    {
#pragma omp single
      { runTaskDag(nf.rootsSN, nf.childrenSN, subtreeWeight, cutoff, forwardProcess); }
    }
    diagonalSolve(nf, Y, Z);
#pragma omp parallel num_threads(requestedThreads)
    {
#pragma omp single
      { runTaskDagTopDown(nf.rootsSN, nf.childrenSN, subtreeWeight, cutoff, backwardProcess); }
    }
    omp_set_max_active_levels(savedMaxActiveLevels);
#endif
  } else {
    // solve.hpp:457-508
    Mat Ywork = Bp;
    for (const auto& f : nf.fronts) {
      const int m = static_cast<int>(f.rowIndices.size());
      const int k = f.nPivots;
      if (k == 0) continue;
      std::vector<double> yOwn(static_cast<size_t>(k) * nrhs);
      for (int p = 0; p < k; ++p)
        for (int c = 0; c < nrhs; ++c) yOwn[p + static_cast<size_t>(c) * k] = Ywork(f.rowIndices[p], c);
      unitLowerSolve(f.Ltop, yOwn.data(), k, nrhs);
      for (int p = 0; p < k; ++p)
        for (int c = 0; c < nrhs; ++c) Ywork(f.rowIndices[p], c) = yOwn[p + static_cast<size_t>(c) * k];
      const int extra = m - k;
      if (extra > 0) {
        for (int c = 0; c < nrhs; ++c)
          for (int i = 0; i < extra; ++i) {
            double s = 0.0;
            for (int p = 0; p < k; ++p) s += f.L(k + i, p) * yOwn[p + static_cast<size_t>(c) * k];
            Ywork(f.rowIndices[k + i], c) -= s;
          }
      }
    }
    Y = std::move(Ywork);
    diagonalSolve(nf, Y, Z);
    for (auto it = nf.fronts.rbegin(); it != nf.fronts.rend(); ++it) {
      const auto& f = *it;
      const int m = static_cast<int>(f.rowIndices.size());
      const int k = f.nPivots;
      if (k == 0) continue;
      std::vector<double> xOwn(static_cast<size_t>(k) * nrhs);
      for (int p = 0; p < k; ++p)
        for (int c = 0; c < nrhs; ++c) xOwn[p + static_cast<size_t>(c) * k] = Z(f.rowIndices[p], c);
      const int extra = m - k;
      if (extra > 0) {
        for (int c = 0; c < nrhs; ++c)
          for (int p = 0; p < k; ++p) {
            double s = 0.0;
            for (int i = 0; i < extra; ++i) s += f.L(k + i, p) * X(f.rowIndices[k + i], c);
            xOwn[p + static_cast<size_t>(c) * k] -= s;
          }
      }
      unitLowerTransSolve(f.Ltop, xOwn.data(), k, nrhs);
      for (int p = 0; p < k; ++p)
        for (int c = 0; c < nrhs; ++c) X(f.rowIndices[p], c) = xOwn[p + static_cast<size_t>(c) * k];
    }
  }
  Mat result(n, nrhs);
  for (int t = 0; t < n; ++t)
    for (int c = 0; c < nrhs; ++c) result(nf.perm[t], c) = X(t, c);
  return result;
}

// ---------------------------------------------------------------------------
// refine.hpp
double sparseMaxAbsRowSum(const Csc& A) {
  std::vector<double> rowAbsSum(A.n, 0.0);
  for (int c = 0; c < A.n; ++c)
    for (int p = A.colptr[c]; p < A.colptr[c + 1]; ++p) rowAbsSum[A.rowind[p]] += std::abs(A.vals[p]);
  double m = 0.0;
  for (double v : rowAbsSum) m = std::max(m, v);
  return m;
}

void symLowerResidual(const Csc& A, const Mat& X, const Mat& B, Mat& R) {
  // R = B - A.selfadjointView<Lower>() * X: the product is formed first,
  // then subtracted (refine.hpp:116).
  const int n = A.n, nrhs = X.cols;
  Mat P(n, nrhs);
  for (int c = 0; c < n; ++c) {
    for (int p = A.colptr[c]; p < A.colptr[c + 1]; ++p) {
      const int r = A.rowind[p];
      if (r < c) continue;  // lower triangle is authoritative
      const double v = A.vals[p];
      for (int k = 0; k < nrhs; ++k) {
        P(r, k) += v * X(c, k);
        if (r != c) P(c, k) += v * X(r, k);
      }
    }
  }
  R = B;
  for (size_t t = 0; t < R.a.size(); ++t) R.a[t] -= P.a[t];
}

namespace {
double infNorm(const Mat& M) {
  // Eigen lpNorm<Infinity>: max |entry|
  double m = 0.0;
  for (double v : M.a) m = std::max(m, std::abs(v));
  return m;
}
}  // namespace

// ---------------------------------------------------------------------------
// solver.hpp
std::vector<int> SymLDLT::buildExpectedSignOriginal(int n) const {
  if (use_explicit_signs) {
    if (static_cast<int>(expected_signs_orig.size()) != n)
      throw std::invalid_argument(
          "symla::SymLDLT::factorize: setExpectedSignPattern's vector size does not match the matrix size");
    return expected_signs_orig;
  }
  std::vector<int> signs(n, 0);
  if (use_kkt_blocks) {
    if (kkt_n1 + kkt_n2 != n)
      throw std::invalid_argument("symla::SymLDLT::factorize: setKKTBlockSizes(n1, n2) sizes do not sum to the matrix size");
    for (int i = 0; i < kkt_n1; ++i) signs[i] = -1;
    for (int i = kkt_n1; i < n; ++i) signs[i] = +1;
  }
  return signs;
}

void SymLDLT::factorize(const Csc& A) {
  attemptDeltas.clear();
  attemptOk.clear();
  if (mode == Mode::StaticRegularized) {
    factorizeStaticRegularized(A);
    return;
  }
  DenseLDLTOptions opts;
  opts.pivot_threshold = pivot_threshold;
  opts.zero_tolerance = zero_tolerance;
  opts.relative_pivot_floor = relative_pivot_floor;
  MultifrontalOptions mf;
  mf.parallel = parallel;
  mf.num_threads = num_threads;
  numeric = multifrontalFactorize(symbolic, A, opts, mf);
  inertia = numeric.inertia;
  factorized = true;
  last_regularization_delta = 0.0;
  regularization_retries_used = 0;
}

void SymLDLT::factorizeStaticRegularized(const Csc& A) {
  const int n = symbolic.n;
  const bool haveExpectation = use_kkt_blocks || use_explicit_signs;
  const std::vector<int> signsOrig = buildExpectedSignOriginal(n);
  std::vector<int> signsFinal(n, 0);
  for (int t = 0; t < n; ++t) signsFinal[t] = signsOrig[symbolic.perm[t]];
  int expectedPos = 0, expectedNeg = 0;
  for (int s : signsOrig) {
    if (s > 0)
      ++expectedPos;
    else if (s < 0)
      ++expectedNeg;
  }
  double delta = initial_regularization_delta;
  if (delta <= 0.0) {
    double maxAbs = 0.0;
    for (int c = 0; c < A.n; ++c)
      for (int p = A.colptr[c]; p < A.colptr[c + 1]; ++p) maxAbs = std::max(maxAbs, std::abs(A.vals[p]));
    if (maxAbs <= 0.0) maxAbs = 1.0;
    delta = std::sqrt(std::numeric_limits<double>::epsilon()) * maxAbs;
  }
  const int maxAttempts = std::max(1, max_regularization_retries + 1);
  for (int attempt = 0; attempt < maxAttempts; ++attempt) {
    DenseLDLTOptions dummy;
    dummy.pivot_threshold = pivot_threshold;
    MultifrontalOptions mf;
    mf.parallel = parallel;
    mf.num_threads = num_threads;
    mf.static_pivoting = true;
    mf.staticOptions.delta = delta;
    mf.staticOptions.relative_pivot_floor = static_pivot_relative_floor;
    mf.staticOptions.absolute_floor = static_pivot_absolute_floor;
    mf.expectedSign = signsFinal;
    NumericFactor attemptResult = multifrontalFactorize(symbolic, A, dummy, mf);
    last_regularization_delta = delta;
    regularization_retries_used = attempt;
    const bool fullCoverage = (expectedPos + expectedNeg == n);
    const bool inertiaOk =
        !haveExpectation ||
        (attemptResult.inertia.n_zero == 0 && !attemptResult.singular &&
         (!fullCoverage || (attemptResult.inertia.n_pos == expectedPos && attemptResult.inertia.n_neg == expectedNeg)));
    attemptDeltas.push_back(delta);
    attemptOk.push_back(inertiaOk ? 1 : 0);
    if (inertiaOk) {
      numeric = std::move(attemptResult);
      inertia = numeric.inertia;
      factorized = true;
      return;
    }
    if (attempt + 1 >= maxAttempts) {
      std::ostringstream oss;
      oss << "symla::SymLDLT::factorize (Mode::StaticRegularized): inertia-controlled regularization retry budget ("
          << max_regularization_retries << " retries) exhausted without matching the expected inertia. expected (n_pos="
          << expectedPos << ", n_neg=" << expectedNeg << ", n_zero=0), got (n_pos=" << attemptResult.inertia.n_pos
          << ", n_neg=" << attemptResult.inertia.n_neg << ", n_zero=" << attemptResult.inertia.n_zero
          << ", singular=" << (attemptResult.singular ? "true" : "false") << ") at delta=" << delta << ".";
      throw std::runtime_error(oss.str());
    }
    delta *= regularization_growth;
  }
}

Mat SymLDLT::solve(const Mat& B) const {
  if (!factorized) throw std::logic_error("symla::SymLDLT::solve: factorize() must be called before solve()");
  if (numeric.singular)
    throw std::logic_error("symla::SymLDLT::solve: factorization is numerically singular; refusing to solve");
  if (B.rows != numeric.n) throw std::invalid_argument("symla::SymLDLT::solve: B.rows() must match the factorized matrix size");
  SolveOptions so;
  so.parallel = parallel;
  so.num_threads = num_threads;
  return multifrontalSolve(numeric, B, so);
}

RefinementResult SymLDLT::solveWithRefinement(const Csc& A, const Mat& B, Mat& X, const RefinementOptions& options) const {
  // solver.hpp:234-240 + refine.hpp:97-144
  X = solve(B);
  RefinementResult result;
  const double normA = sparseMaxAbsRowSum(A);
  const double normB = infNorm(B);
  auto relResidual = [&](const Mat& R, const Mat& Xc) {
    const double normR = infNorm(R);
    const double normX = infNorm(Xc);
    const double denom = normA * normX + normB;
    return denom > 0.0 ? normR / denom : normR;
  };
  Mat R;
  symLowerResidual(A, X, B, R);
  double res = relResidual(R, X);
  result.initial_relative_residual = res;
  result.final_relative_residual = res;
  for (int it = 0; it < options.max_iterations; ++it) {
    if (res <= options.tolerance) break;
    Mat dx = solve(R);
    Mat Xnew = X;
    for (size_t t = 0; t < Xnew.a.size(); ++t) Xnew.a[t] += dx.a[t];
    Mat Rnew;
    symLowerResidual(A, Xnew, B, Rnew);
    const double resNew = relResidual(Rnew, Xnew);
    if (!(resNew < res)) break;
    X = std::move(Xnew);
    R = std::move(Rnew);
    res = resNew;
    result.iterations = it + 1;
    result.final_relative_residual = res;
  }
  return result;
}

}  // namespace oracle
