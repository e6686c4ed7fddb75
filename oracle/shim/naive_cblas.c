/*
 * Deterministic CBLAS subset (column-major only) for building the reference's
 * own AM solver in oracle/_ref/.  Test infrastructure only.
 *
 * Every reduction runs sequentially in index order in the routine's own
 * precision, so results do not depend on thread count or CPU.  The oracle's C
 * restatement (oracle/am_oracle.c) uses the same summation order, which makes
 * the two bit-identical on the same inputs.
 */
#include <math.h>
#include "gsl/gsl_cblas.h"

#define DEF_GEMM(NAME, T)                                                               \
  void NAME(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,            \
            const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,   \
            const T alpha, const T *A, const int lda, const T *B, const int ldb,        \
            const T beta, T *C, const int ldc) {                                        \
    (void)Order;                                                                        \
    for (int j = 0; j < N; j++) {                                                       \
      for (int i = 0; i < M; i++) {                                                     \
        T acc = 0;                                                                      \
        for (int l = 0; l < K; l++) {                                                   \
          T a = (TransA == CblasNoTrans) ? A[i + (long)l * lda] : A[l + (long)i * lda]; \
          T b = (TransB == CblasNoTrans) ? B[l + (long)j * ldb] : B[j + (long)l * ldb]; \
          acc += a * b;                                                                 \
        }                                                                               \
        T *c = &C[i + (long)j * ldc];                                                   \
        *c = (beta == 0) ? alpha * acc : alpha * acc + beta * *c;                       \
      }                                                                                 \
    }                                                                                   \
  }
DEF_GEMM(cblas_sgemm, float)
DEF_GEMM(cblas_dgemm, double)

#define DEF_VEC(S, T)                                                                   \
  void cblas_##S##scal(const int N, const T alpha, T *X, const int incX) {              \
    for (int i = 0; i < N; i++) X[(long)i * incX] *= alpha;                              \
  }                                                                                     \
  T cblas_##S##asum(const int N, const T *X, const int incX) {                          \
    T s = 0;                                                                            \
    for (int i = 0; i < N; i++) s += (X[(long)i * incX] < 0 ? -X[(long)i * incX]        \
                                                             : X[(long)i * incX]);      \
    return s;                                                                           \
  }                                                                                     \
  T cblas_##S##nrm2(const int N, const T *X, const int incX) {                          \
    T s = 0;                                                                            \
    for (int i = 0; i < N; i++) s += X[(long)i * incX] * X[(long)i * incX];             \
    return (T)sqrt((double)s);                                                          \
  }                                                                                     \
  void cblas_##S##copy(const int N, const T *X, const int incX, T *Y, const int incY) { \
    for (int i = 0; i < N; i++) Y[(long)i * incY] = X[(long)i * incX];                  \
  }                                                                                     \
  CBLAS_INDEX cblas_i##S##amax(const int N, const T *X, const int incX) {               \
    CBLAS_INDEX best = 0;                                                               \
    T bv = -1;                                                                          \
    for (int i = 0; i < N; i++) {                                                       \
      T v = X[(long)i * incX];                                                          \
      v = v < 0 ? -v : v;                                                               \
      if (v > bv) { bv = v; best = (CBLAS_INDEX)i; }                                    \
    }                                                                                   \
    return best;                                                                        \
  }
DEF_VEC(s, float)
DEF_VEC(d, double)
