// ORACLE -- test infrastructure only (see oracle.hpp).
// C -= X * Y^T for the trailing update of the dense kernel (the reference
// evaluates `trailing -= Lpanel * Dpanel * Lpanel^T` with Eigen's GEMM,
// dense_kernel.hpp:817 and :1050). Like Eigen's GEMM it packs its operands
// into cache-resident panels and runs a register-blocked micro-kernel with
// fused multiply-adds (this file is compiled with FMA contraction allowed;
// everything else in the oracle with -ffp-contract=off, CMakeLists.txt:92-127).
// Like Eigen's GEMM under OpenMP it runs on one thread inside a parallel
// region (the reference pins Eigen to one thread there,
// multifrontal.hpp:732-733) and splits the columns over the team outside one.
#include <omp.h>

#include <algorithm>
#include <cstddef>
#include <vector>

#include "oracle.hpp"

namespace oracle {

namespace {

typedef double v8d __attribute__((vector_size(64)));

constexpr int kMR = 16;   // rows of a micro-tile (two 8-wide vectors)
constexpr int kNR = 8;    // columns of a micro-tile
constexpr int kMC = 192;  // rows of a packed X block (kMC * p doubles stay in L2)

inline v8d load8(const double* p) {
  v8d v;
  __builtin_memcpy(&v, p, sizeof(v));
  return v;
}
inline void store8(double* p, v8d v) { __builtin_memcpy(p, &v, sizeof(v)); }

// acc(16 x 8) = Xp(16 x p) * Yp(8 x p)^T with Xp packed k-major (16 per k)
// and Yp packed k-major (8 per k); then C(0:mr, 0:nr) -= acc.
void microKernel(int p, const double* Xp, const double* Yp, double* C, int ldc, int mr, int nr) {
  v8d a[2][kNR];
  for (int j = 0; j < kNR; ++j) a[0][j] = a[1][j] = v8d{0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < p; ++k) {
    const v8d x0 = load8(Xp + static_cast<size_t>(k) * kMR);
    const v8d x1 = load8(Xp + static_cast<size_t>(k) * kMR + 8);
    const double* y = Yp + static_cast<size_t>(k) * kNR;
#pragma GCC unroll 8
    for (int j = 0; j < kNR; ++j) {
      a[0][j] += x0 * y[j];
      a[1][j] += x1 * y[j];
    }
  }
  if (mr == kMR) {
    for (int j = 0; j < nr; ++j) {
      double* c = C + static_cast<size_t>(j) * ldc;
      store8(c, load8(c) - a[0][j]);
      store8(c + 8, load8(c + 8) - a[1][j]);
    }
  } else {
    alignas(64) double t[kMR];
    for (int j = 0; j < nr; ++j) {
      double* c = C + static_cast<size_t>(j) * ldc;
      store8(t, a[0][j]);
      store8(t + 8, a[1][j]);
      for (int i = 0; i < mr; ++i) c[i] -= t[i];
    }
  }
}

void packX(int mc, int p, const double* X, int ldx, double* Xp) {
  for (int ib = 0; ib < mc; ib += kMR) {
    const int mr = std::min(kMR, mc - ib);
    double* dst = Xp + static_cast<size_t>(ib) * p;
    for (int k = 0; k < p; ++k) {
      const double* src = X + ib + static_cast<size_t>(k) * ldx;
      double* d = dst + static_cast<size_t>(k) * kMR;
      int i = 0;
      for (; i < mr; ++i) d[i] = src[i];
      for (; i < kMR; ++i) d[i] = 0.0;
    }
  }
}

void packY(int cols, int p, const double* Y, int ldy, double* Yp) {
  for (int jb = 0; jb < cols; jb += kNR) {
    const int nr = std::min(kNR, cols - jb);
    double* dst = Yp + static_cast<size_t>(jb) * p;
    for (int k = 0; k < p; ++k) {
      const double* src = Y + jb + static_cast<size_t>(k) * ldy;
      double* d = dst + static_cast<size_t>(k) * kNR;
      int j = 0;
      for (; j < nr; ++j) d[j] = src[j];
      for (; j < kNR; ++j) d[j] = 0.0;
    }
  }
}

// Columns [c0, c1) of C -= X * Y^T (c0, c1 multiples of kNR or c1 = rows).
void gemmColumns(int rows, int c0, int c1, int p, const double* X, int ldx, const double* Yp, double* C, int ldc,
                 std::vector<double>& xbuf) {
  xbuf.resize(static_cast<size_t>(kMC) * p);
  for (int i0 = 0; i0 < rows; i0 += kMC) {
    const int mc = std::min(kMC, rows - i0);
    packX(mc, p, X + i0, ldx, xbuf.data());
    for (int jb = c0; jb < c1; jb += kNR) {
      const int nr = std::min(kNR, c1 - jb);
      const double* yp = Yp + static_cast<size_t>(jb) * p;
      for (int ib = 0; ib < mc; ib += kMR) {
        microKernel(p, xbuf.data() + static_cast<size_t>(ib) * p, yp,
                    C + (i0 + ib) + static_cast<size_t>(jb) * ldc, ldc, std::min(kMR, mc - ib), nr);
      }
    }
  }
}

}  // namespace

void gemmSubNT(int rows, int p, const double* X, int ldx, const double* Y, int ldy, double* C, int ldc) {
  if (rows <= 0 || p <= 0) return;
  static thread_local std::vector<double> ybuf, xbuf;
  ybuf.resize(static_cast<size_t>((rows + kNR - 1) / kNR) * kNR * p);
  packY(rows, p, Y, ldy, ybuf.data());
  const double work = 2.0 * rows * static_cast<double>(rows) * p;
  const int team = omp_in_parallel() ? 1 : omp_get_max_threads();
  if (team > 1 && work > 5e7) {
    const int nblk = (rows + kNR - 1) / kNR;
    const double* yp = ybuf.data();
#pragma omp parallel num_threads(team)
    {
      static thread_local std::vector<double> xb;
      const int t = omp_get_thread_num(), nt = omp_get_num_threads();
      const int b0 = static_cast<int>(static_cast<long long>(nblk) * t / nt);
      const int b1 = static_cast<int>(static_cast<long long>(nblk) * (t + 1) / nt);
      if (b1 > b0) gemmColumns(rows, b0 * kNR, std::min(rows, b1 * kNR), p, X, ldx, yp, C, ldc, xb);
    }
  } else {
    gemmColumns(rows, 0, rows, p, X, ldx, ybuf.data(), C, ldc, xbuf);
  }
}

}  // namespace oracle
