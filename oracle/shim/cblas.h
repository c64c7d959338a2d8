/*
 * Minimal row-major CBLAS used to compile the DynELA reference sources as a CPU
 * oracle (test infrastructure only).  No CBLAS library is installed in this
 * image; the reference calls cblas_dgemm for dN/dx = dN/dxi . J^-1 on every
 * Jacobian (Sources/dnlMaths/Matrix.C:815) and cblas_dgemv off the hot path
 * (Matrix.C:1000-1071).  The products are straightforward triple loops with a
 * left-to-right sum over k, which is the arithmetic the engine reproduces.
 */
#ifndef DNL_ORACLE_CBLAS_SHIM_H
#define DNL_ORACLE_CBLAS_SHIM_H

#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

static inline double dnl_shim_elem(const double *m, int ld, int trans, int i, int j, int rowmajor)
{
  /* element (i, j) of op(M) */
  if (trans) { int t = i; i = j; j = t; }
  return rowmajor ? m[(long)i * ld + j] : m[(long)j * ld + i];
}

static inline void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                               int M, int N, int K, double alpha, const double *A, int lda,
                               const double *B, int ldb, double beta, double *C, int ldc)
{
  int rm = (order == CblasRowMajor);
  for (int i = 0; i < M; i++)
    for (int j = 0; j < N; j++)
    {
      double s = 0.0;
      for (int k = 0; k < K; k++)
        s += dnl_shim_elem(A, lda, ta != CblasNoTrans, i, k, rm) * dnl_shim_elem(B, ldb, tb != CblasNoTrans, k, j, rm);
      double *c = rm ? &C[(long)i * ldc + j] : &C[(long)j * ldc + i];
      *c = (beta == 0.0) ? alpha * s : alpha * s + beta * (*c);
    }
}

static inline void cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, int M, int N, double alpha,
                               const double *A, int lda, const double *x, int incx, double beta, double *y, int incy)
{
  int rm = (order == CblasRowMajor);
  int tr = (ta != CblasNoTrans);
  int rows = tr ? N : M, cols = tr ? M : N;
  for (int i = 0; i < rows; i++)
  {
    double s = 0.0;
    for (int k = 0; k < cols; k++)
    {
      /* op(A)(i,k) where A is M x N */
      double a = tr ? (rm ? A[(long)k * lda + i] : A[(long)i * lda + k]) : (rm ? A[(long)i * lda + k] : A[(long)k * lda + i]);
      s += a * x[(long)k * incx];
    }
    double *yy = &y[(long)i * incy];
    *yy = (beta == 0.0) ? alpha * s : alpha * s + beta * (*yy);
  }
}

#ifdef __cplusplus
}
#endif

#endif
