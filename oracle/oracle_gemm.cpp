// ORACLE -- test infrastructure only (see oracle.hpp).
// Register-blocked C -= X * Y^T used for the trailing update of the dense
// kernel (the reference evaluates `trailing -= Lpanel * Dpanel * Lpanel^T`
// with Eigen's GEMM, dense_kernel.hpp:817 and :1050). Compiled with FMA
// contraction allowed, like Eigen's packet GEMM; everything else in the
// oracle is compiled with -ffp-contract=off (CMakeLists.txt:92-127).
#include <cstddef>

#include "oracle.hpp"

namespace oracle {

typedef double v8d __attribute__((vector_size(64)));

void gemmSubNT(int rows, int p, const double* X, int ldx, const double* Y, int ldy, double* C, int ldc) {
  if (rows <= 0 || p <= 0) return;
  const int i8 = rows & ~7;
  const int j4 = rows & ~3;
  for (int j = 0; j < j4; j += 4) {
    double* c0 = C + static_cast<size_t>(j) * ldc;
    double* c1 = c0 + ldc;
    double* c2 = c1 + ldc;
    double* c3 = c2 + ldc;
    for (int i = 0; i < i8; i += 8) {
      v8d a0 = {0, 0, 0, 0, 0, 0, 0, 0}, a1 = a0, a2 = a0, a3 = a0;
      for (int k = 0; k < p; ++k) {
        v8d x;
        __builtin_memcpy(&x, X + i + static_cast<size_t>(k) * ldx, sizeof(x));
        const double* yk = Y + static_cast<size_t>(k) * ldy + j;
        a0 += x * yk[0];
        a1 += x * yk[1];
        a2 += x * yk[2];
        a3 += x * yk[3];
      }
      v8d t;
      __builtin_memcpy(&t, c0 + i, sizeof(t));
      t -= a0;
      __builtin_memcpy(c0 + i, &t, sizeof(t));
      __builtin_memcpy(&t, c1 + i, sizeof(t));
      t -= a1;
      __builtin_memcpy(c1 + i, &t, sizeof(t));
      __builtin_memcpy(&t, c2 + i, sizeof(t));
      t -= a2;
      __builtin_memcpy(c2 + i, &t, sizeof(t));
      __builtin_memcpy(&t, c3 + i, sizeof(t));
      t -= a3;
      __builtin_memcpy(c3 + i, &t, sizeof(t));
    }
    for (int i = i8; i < rows; ++i) {
      double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
      for (int k = 0; k < p; ++k) {
        const double x = X[i + static_cast<size_t>(k) * ldx];
        const double* yk = Y + static_cast<size_t>(k) * ldy + j;
        s0 += x * yk[0];
        s1 += x * yk[1];
        s2 += x * yk[2];
        s3 += x * yk[3];
      }
      c0[i] -= s0;
      c1[i] -= s1;
      c2[i] -= s2;
      c3[i] -= s3;
    }
  }
  for (int j = j4; j < rows; ++j) {
    double* cj = C + static_cast<size_t>(j) * ldc;
    for (int i = 0; i < rows; ++i) {
      double s = 0;
      for (int k = 0; k < p; ++k) s += X[i + static_cast<size_t>(k) * ldx] * Y[j + static_cast<size_t>(k) * ldy];
      cj[i] -= s;
    }
  }
}

}  // namespace oracle
