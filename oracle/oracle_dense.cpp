// ORACLE -- test infrastructure only (see oracle.hpp).
// Restatement of include/symla/dense_kernel.hpp (DenseLDLT::factor,
// DenseLDLT::factorStatic, resymmetrizeTrailingTiled).
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <vector>

#include "oracle.hpp"

namespace oracle {

namespace {

// dense_kernel.hpp:269-297 -- average both triangles of the trailing block in
// 64x64 tiles (order-independent per entry).
void resymmetrizeTrailingTiled(MatView T) {
  const int extent = T.rows;
  if (extent == 0) return;
  constexpr int kTile = 64;
  for (int jb = 0; jb < extent; jb += kTile) {
    const int jn = std::min(kTile, extent - jb);
    for (int ib = jb; ib < extent; ib += kTile) {
      const int in = std::min(kTile, extent - ib);
      if (ib == jb) {
        for (int j = jb; j < jb + jn; ++j)
          for (int i = j + 1; i < jb + jn; ++i) {
            const double avg = 0.5 * (T(i, j) + T(j, i));
            T(i, j) = avg;
            T(j, i) = avg;
          }
      } else {
        for (int j = jb; j < jb + jn; ++j)
          for (int i = ib; i < ib + in; ++i) {
            const double avg = 0.5 * (T(i, j) + T(j, i));
            T(i, j) = avg;
            T(j, i) = avg;
          }
      }
    }
  }
}

double maxAbsBlock(const MatView& A, int r0, int c0, int nr, int nc) {
  double m = 0.0;
  for (int j = 0; j < nc; ++j)
    for (int i = 0; i < nr; ++i) m = std::max(m, std::abs(A(r0 + i, c0 + j)));
  return m;
}

// LD = Lblk * Dp for the p x p block-diagonal Dp (1x1 / 2x2 blocks), Lblk
// rows x p. Only structurally nonzero entries of Dp contribute.
void timesBlockDiag(const double* L, int ldl, int rows, int p, const BlockDiagonalD& Dbuf, double* LD) {
  for (int j = 0; j < p; ++j) {
    const double dj = Dbuf.diag[j];
    const double offPrev = (j > 0) ? Dbuf.offdiag[j - 1] : 0.0;  // Dp(j-1, j)
    const double offNext = (j + 1 < p) ? Dbuf.offdiag[j] : 0.0;  // Dp(j+1, j)
    for (int i = 0; i < rows; ++i) {
      double v = L[i + static_cast<size_t>(j) * ldl] * dj;
      if (offPrev != 0.0) v += L[i + static_cast<size_t>(j - 1) * ldl] * offPrev;
      if (offNext != 0.0) v += L[i + static_cast<size_t>(j + 1) * ldl] * offNext;
      LD[i + static_cast<size_t>(j) * rows] = v;
    }
  }
}

}  // namespace

DenseLDLTResult denseFactor(MatView A, BlockDiagonalD& D_out, const DenseLDLTOptions& options, int n_eligible) {
  const int n = A.rows;
  if (A.cols != n) throw std::invalid_argument("DenseLDLT::factor: A must be square");
  const int effEnd = (n_eligible < 0) ? n : n_eligible;
  if (effEnd < 0 || effEnd > n) throw std::invalid_argument("DenseLDLT::factor: n_eligible out of range");

  const double alpha = (1.0 + std::sqrt(17.0)) / 8.0;
  const int panelSizeOpt = options.panel_size > 0 ? options.panel_size : 64;

  DenseLDLTResult result;
  result.perm.resize(n);
  for (int i = 0; i < n; ++i) result.perm[i] = i;
  D_out.resize(n);

  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) A(j, i) = A(i, j);

  double orig_max = maxAbsBlock(A, 0, 0, n, n);
  if (orig_max < options.zero_tolerance) orig_max = 1.0;
  double running_max = orig_max;

  auto swap_rowcol = [&](int i, int j) {
    if (i == j) return;
    for (int c = 0; c < n; ++c) std::swap(A(i, c), A(j, c));
    for (int r = 0; r < n; ++r) std::swap(A(r, i), A(r, j));
    std::swap(result.perm[i], result.perm[j]);
  };

  int k = 0;
  std::vector<double> LDtmp, corr;
  while (k < effEnd) {
    const int panelStart = k;
    const int panelWidthTarget = std::min(panelSizeOpt, effEnd - panelStart);
    const int panelEnd = panelStart + panelWidthTarget;
    const int panelCapacity = panelWidthTarget + 1;
    const int m0 = n - panelStart;

    Mat Lbuf(m0, panelCapacity);
    BlockDiagonalD Dbuf;
    Dbuf.resize(panelCapacity);
    Mat Araw(m0, m0);
    for (int j = 0; j < m0; ++j)
      for (int i = 0; i < m0; ++i) Araw(i, j) = A(panelStart + i, panelStart + j);
    std::vector<int> appliedCount(m0, 0);
    bool panelStoppedEarly = false;

    // dense_kernel.hpp:516-545
    auto setColumnRaw = [&](int col, int p) {
      const int idx = col - panelStart;
      const int rowsFrom = k - panelStart;
      const int rowsCount = m0 - rowsFrom;
      if (rowsCount <= 0) {
        appliedCount[idx] = p;
        return;
      }
      if (p == 0) {
        for (int t = 0; t < rowsCount; ++t) A(k + t, col) = Araw(rowsFrom + t, idx);
      } else {
        LDtmp.assign(static_cast<size_t>(rowsCount) * p, 0.0);
        timesBlockDiag(&Lbuf(rowsFrom, 0), Lbuf.rows, rowsCount, p, Dbuf, LDtmp.data());
        corr.assign(rowsCount, 0.0);
        for (int j = 0; j < p; ++j) {
          const double lr = Lbuf(idx, j);
          const double* ldc = &LDtmp[static_cast<size_t>(j) * rowsCount];
          for (int t = 0; t < rowsCount; ++t) corr[t] += ldc[t] * lr;
        }
        for (int t = 0; t < rowsCount; ++t) A(k + t, col) = Araw(rowsFrom + t, idx) - corr[t];
      }
      for (int t = 0; t < rowsCount; ++t) A(col, k + t) = A(k + t, col);
      appliedCount[idx] = p;
    };
    auto ensureColumnCurrent = [&](int col, int p) {
      if (appliedCount[col - panelStart] == p) return;
      setColumnRaw(col, p);
    };
    // dense_kernel.hpp:565-573
    auto panelSwap = [&](int i, int j) {
      if (i == j) return;
      swap_rowcol(i, j);
      const int ii = i - panelStart, jj = j - panelStart;
      for (int c = 0; c < panelCapacity; ++c) std::swap(Lbuf(ii, c), Lbuf(jj, c));
      for (int c = 0; c < m0; ++c) std::swap(Araw(ii, c), Araw(jj, c));
      for (int r = 0; r < m0; ++r) std::swap(Araw(r, ii), Araw(r, jj));
      std::swap(appliedCount[ii], appliedCount[jj]);
    };
    auto recordOneByOne = [&](int p) {
      const int m = n - k;
      running_max = std::max(running_max, std::abs(A(k, k)));
      const double d = A(k, k);
      D_out.diag[k] = d;
      Dbuf.diag[p] = d;
      result.pivots.push_back({k, PivotKind::OneByOne});
      if (d > 0)
        ++result.inertia.n_pos;
      else if (d < 0)
        ++result.inertia.n_neg;
      else
        ++result.inertia.n_zero;
      if (m > 1) {
        running_max = std::max(running_max, maxAbsBlock(A, k + 1, k, m - 1, 1));
        for (int t = 1; t < m; ++t) {
          const double l = A(k + t, k) / d;
          Lbuf(k + t - panelStart, p) = l;
          A(k + t, k) = l;
          A(k, k + t) = l;
        }
      }
    };

    int p = 0;
    while (k < panelEnd) {
      ensureColumnCurrent(k, p);

      double lambda = 0.0;
      int r = -1;
      for (int i = k + 1; i < effEnd; ++i) {
        const double v = std::abs(A(i, k));
        if (v > lambda) {
          lambda = v;
          r = i;
        }
      }

      bool accept_1x1_at_k = false;
      bool accept_1x1_swap_kr = false;
      if (lambda <= options.zero_tolerance) {
        const double isolatedFloor = std::max(options.zero_tolerance, options.relative_pivot_floor * orig_max);
        if (std::abs(A(k, k)) <= isolatedFloor) {
          panelStoppedEarly = true;
          break;
        }
        accept_1x1_at_k = true;
      } else if (std::abs(A(k, k)) >= alpha * lambda) {
        accept_1x1_at_k = true;
      } else {
        ensureColumnCurrent(r, p);
        double sigma = 0.0;
        for (int i = k; i < effEnd; ++i) {
          if (i == r) continue;
          const double v = std::abs(A(i, r));
          if (v > sigma) sigma = v;
        }
        if (std::abs(A(k, k)) * sigma >= alpha * lambda * lambda) {
          accept_1x1_at_k = true;
        } else if (std::abs(A(r, r)) >= alpha * sigma) {
          accept_1x1_swap_kr = true;
        }
      }

      if (accept_1x1_at_k) {
        recordOneByOne(p);
        ++k;
        ++p;
        continue;
      }
      if (accept_1x1_swap_kr) {
        panelSwap(k, r);
        recordOneByOne(p);
        ++k;
        ++p;
        continue;
      }
      // 2x2 pivot at (k, r)
      {
        if (r != k + 1) panelSwap(k + 1, r);
        const double d11 = A(k, k);
        const double d21 = A(k + 1, k);
        const double d22 = A(k + 1, k + 1);
        const double det = d11 * d22 - d21 * d21;
        if (std::abs(det) <=
            options.zero_tolerance * std::max(1.0, running_max) * std::max(1.0, running_max)) {
          panelStoppedEarly = true;
          break;
        }
        running_max = std::max(running_max, std::max({std::abs(d11), std::abs(d21), std::abs(d22)}));
        D_out.diag[k] = d11;
        D_out.offdiag[k] = d21;
        D_out.diag[k + 1] = d22;
        Dbuf.diag[p] = d11;
        Dbuf.offdiag[p] = d21;
        Dbuf.diag[p + 1] = d22;
        result.pivots.push_back({k, PivotKind::TwoByTwo});
        if (det < 0) {
          ++result.inertia.n_pos;
          ++result.inertia.n_neg;
        } else {
          const double tr = d11 + d22;
          if (tr > 0)
            result.inertia.n_pos += 2;
          else if (tr < 0)
            result.inertia.n_neg += 2;
          else {
            ++result.inertia.n_pos;
            ++result.inertia.n_neg;
          }
        }
        const int mm = n - (k + 2);
        if (mm > 0) {
          const double inv11 = d22 / det;
          const double inv21 = -d21 / det;
          const double inv22 = d11 / det;
          running_max = std::max(running_max, maxAbsBlock(A, k + 2, k, mm, 2));
          for (int t = 0; t < mm; ++t) {
            const double a0 = A(k + 2 + t, k), a1 = A(k + 2 + t, k + 1);
            const double l0 = a0 * inv11 + a1 * inv21;
            const double l1 = a0 * inv21 + a1 * inv22;
            Lbuf(k + 2 + t - panelStart, p) = l0;
            Lbuf(k + 2 + t - panelStart, p + 1) = l1;
            A(k + 2 + t, k) = l0;
            A(k + 2 + t, k + 1) = l1;
            A(k, k + 2 + t) = l0;
            A(k + 1, k + 2 + t) = l1;
          }
        }
        k += 2;
        p += 2;
        continue;
      }
    }

    // dense_kernel.hpp:806-821
    if (p > 0) {
      for (int col = k; col < n; ++col)
        if (appliedCount[col - panelStart] != 0) setColumnRaw(col, 0);
      const int rowsCount = n - k;
      if (rowsCount > 0) {
        std::vector<double> LD(static_cast<size_t>(rowsCount) * p);
        timesBlockDiag(&Lbuf(k - panelStart, 0), Lbuf.rows, rowsCount, p, Dbuf, LD.data());
        gemmSubNT(rowsCount, p, LD.data(), rowsCount, &Lbuf(k - panelStart, 0), Lbuf.rows, &A(k, k), A.ld);
        MatView T{&A(k, k), rowsCount, rowsCount, A.ld};
        resymmetrizeTrailingTiled(T);
        running_max = std::max(running_max, maxAbsBlock(T, 0, 0, rowsCount, rowsCount));
      }
    }
    if (panelStoppedEarly) break;
  }

  result.n_factored = k;
  for (int j = k; j < effEnd; ++j) result.delayed_cols.push_back(j);
  result.max_growth = running_max / orig_max;
  return result;
}

DenseLDLTResult denseFactorStatic(MatView A, BlockDiagonalD& D_out, const StaticPivotOptions& options,
                                  const std::vector<int>& expectedSign, int n_eligible) {
  const int n = A.rows;
  if (A.cols != n) throw std::invalid_argument("DenseLDLT::factorStatic: A must be square");
  const int effEnd = (n_eligible < 0) ? n : n_eligible;
  if (effEnd < 0 || effEnd > n) throw std::invalid_argument("DenseLDLT::factorStatic: n_eligible out of range");

  DenseLDLTResult result;
  result.perm.resize(n);
  for (int i = 0; i < n; ++i) result.perm[i] = i;
  D_out.resize(n);
  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) A(j, i) = A(i, j);

  double orig_max = maxAbsBlock(A, 0, 0, n, n);
  if (orig_max < options.absolute_floor) orig_max = 1.0;
  double running_max = orig_max;
  const double delta =
      options.delta > 0.0 ? options.delta : std::sqrt(std::numeric_limits<double>::epsilon()) * orig_max;
  const double floor = std::max(options.absolute_floor, options.relative_pivot_floor * orig_max);
  const int panelSizeOpt = options.panel_size > 0 ? options.panel_size : 64;

  int k = 0;
  std::vector<double> col, Dl;
  while (k < effEnd) {
    const int panelStart = k;
    const int panelWidth = std::min(panelSizeOpt, effEnd - panelStart);
    const int panelEnd = panelStart + panelWidth;
    const int m0 = n - panelStart;
    Mat Araw(m0, panelWidth);
    for (int j = 0; j < panelWidth; ++j)
      for (int i = 0; i < m0; ++i) Araw(i, j) = A(panelStart + i, panelStart + j);
    Mat Lbuf(m0, panelWidth);
    std::vector<double> Dbuf(panelWidth, 0.0);

    for (; k < panelEnd; ++k) {
      const int idx = k - panelStart;
      const int rowsCount = m0 - idx;
      col.assign(rowsCount, 0.0);
      if (idx == 0) {
        for (int t = 0; t < rowsCount; ++t) col[t] = Araw(t, 0);
      } else {
        Dl.assign(idx, 0.0);
        for (int j = 0; j < idx; ++j) Dl[j] = Lbuf(idx, j) * Dbuf[j];
        for (int t = 0; t < rowsCount; ++t) col[t] = 0.0;
        for (int j = 0; j < idx; ++j) {
          const double dl = Dl[j];
          for (int t = 0; t < rowsCount; ++t) col[t] += Lbuf(idx + t, j) * dl;
        }
        for (int t = 0; t < rowsCount; ++t) col[t] = Araw(idx + t, idx) - col[t];
      }
      const double a_kk = col[0];
      const int sign = (k < static_cast<int>(expectedSign.size())) ? expectedSign[k] : 0;
      double d = a_kk;
      double applied = 0.0;
      bool needPerturb;
      if (sign > 0)
        needPerturb = a_kk < floor;
      else if (sign < 0)
        needPerturb = a_kk > -floor;
      else
        needPerturb = std::abs(a_kk) < floor;
      if (needPerturb) {
        const double s = (sign != 0) ? static_cast<double>(sign) : (a_kk >= 0.0 ? 1.0 : -1.0);
        d = a_kk + s * delta;
        applied = d - a_kk;
      }
      D_out.diag[k] = d;
      Dbuf[idx] = d;
      result.pivots.push_back({k, PivotKind::OneByOne});
      if (applied != 0.0) {
        result.total_perturbation += std::abs(applied);
        ++result.num_perturbed;
      }
      if (d > 0)
        ++result.inertia.n_pos;
      else if (d < 0)
        ++result.inertia.n_neg;
      else
        ++result.inertia.n_zero;
      running_max = std::max(running_max, std::abs(d));
      if (rowsCount > 1) {
        double mx = 0.0;
        for (int t = 1; t < rowsCount; ++t) mx = std::max(mx, std::abs(col[t]));
        running_max = std::max(running_max, mx);
        for (int t = 1; t < rowsCount; ++t) {
          const double l = col[t] / d;
          Lbuf(idx + t, idx) = l;
          A(k + t, k) = l;
          A(k, k + t) = l;
        }
      }
    }
    const int rowsBeyond = n - panelEnd;
    if (rowsBeyond > 0) {
      const int off = panelEnd - panelStart;
      std::vector<double> LD(static_cast<size_t>(rowsBeyond) * panelWidth);
      for (int j = 0; j < panelWidth; ++j)
        for (int t = 0; t < rowsBeyond; ++t)
          LD[t + static_cast<size_t>(j) * rowsBeyond] = Lbuf(off + t, j) * Dbuf[j];
      gemmSubNT(rowsBeyond, panelWidth, LD.data(), rowsBeyond, &Lbuf(off, 0), Lbuf.rows, &A(panelEnd, panelEnd),
                A.ld);
      MatView T{&A(panelEnd, panelEnd), rowsBeyond, rowsBeyond, A.ld};
      resymmetrizeTrailingTiled(T);
      running_max = std::max(running_max, maxAbsBlock(T, 0, 0, rowsBeyond, rowsBeyond));
    }
  }
  result.n_factored = effEnd;
  result.max_growth = running_max / orig_max;
  return result;
}

}  // namespace oracle
