/*
 * Minimal CBLAS declarations, written for this project as TEST INFRASTRUCTURE.
 *
 * The reference's sparse containers include its dense-GEMM wrapper, which
 * needs <cblas.h> to compile even though the sparse tile multiply never calls
 * it.  These naive row/column-major loops satisfy the two symbols it names.
 */
#ifndef BCLX_CBLAS_STUB_H
#define BCLX_CBLAS_STUB_H

#include <stddef.h>

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

#define BCLX_CBLAS_GEMM(NAME, T)                                                        \
  static inline void NAME(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,        \
                          int m, int n, int k, T alpha, const T* a, int lda,            \
                          const T* b, int ldb, T beta, T* c, int ldc) {                 \
    for (int i = 0; i < m; i++)                                                         \
      for (int j = 0; j < n; j++) {                                                     \
        T acc = 0;                                                                      \
        for (int p = 0; p < k; p++) {                                                   \
          T av, bv;                                                                     \
          if (o == CblasRowMajor) {                                                     \
            av = (ta == CblasNoTrans) ? a[(size_t)i * lda + p] : a[(size_t)p * lda + i]; \
            bv = (tb == CblasNoTrans) ? b[(size_t)p * ldb + j] : b[(size_t)j * ldb + p]; \
          } else {                                                                      \
            av = (ta == CblasNoTrans) ? a[(size_t)p * lda + i] : a[(size_t)i * lda + p]; \
            bv = (tb == CblasNoTrans) ? b[(size_t)j * ldb + p] : b[(size_t)p * ldb + j]; \
          }                                                                             \
          acc += av * bv;                                                               \
        }                                                                               \
        T* cp = (o == CblasRowMajor) ? &c[(size_t)i * ldc + j] : &c[(size_t)j * ldc + i]; \
        *cp = alpha * acc + beta * *cp;                                                 \
      }                                                                                 \
  }

BCLX_CBLAS_GEMM(cblas_sgemm, float)
BCLX_CBLAS_GEMM(cblas_dgemm, double)

#undef BCLX_CBLAS_GEMM

#endif
