/*
 * LAPACKE stand-in used to compile the DynELA reference sources as a CPU oracle
 * (test infrastructure only).  LAPACKE is not installed in this image and the
 * reference only calls it off the per-increment path (matrix inverses, SVD and
 * the LAPACK polar-decomposition variants: Matrix.C:1461-2106,
 * Tensor2.C:1560,1662, SymTensor2.C:1440,1542).  Every function here aborts, so
 * a test that reached one would fail loudly instead of computing something else.
 */
#ifndef DNL_ORACLE_LAPACKE_SHIM_H
#define DNL_ORACLE_LAPACKE_SHIM_H

#include <stdio.h>
#include <stdlib.h>

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

#define DNL_SHIM_ABORT(name) \
  do { fprintf(stderr, "oracle: LAPACKE function %s is not available\n", name); abort(); } while (0)

#ifdef __cplusplus
extern "C" {
#endif
static inline lapack_int LAPACKE_dgetrf(int, lapack_int, lapack_int, double *, lapack_int, lapack_int *) { DNL_SHIM_ABORT("dgetrf"); return -1; }
static inline lapack_int LAPACKE_dgetri(int, lapack_int, double *, lapack_int, const lapack_int *) { DNL_SHIM_ABORT("dgetri"); return -1; }
static inline lapack_int LAPACKE_dgesv(int, lapack_int, lapack_int, double *, lapack_int, lapack_int *, double *, lapack_int) { DNL_SHIM_ABORT("dgesv"); return -1; }
static inline lapack_int LAPACKE_dgesvd(int, char, char, lapack_int, lapack_int, double *, lapack_int, double *, double *, lapack_int, double *, lapack_int, double *) { DNL_SHIM_ABORT("dgesvd"); return -1; }
static inline lapack_int LAPACKE_dgesdd(int, char, lapack_int, lapack_int, double *, lapack_int, double *, double *, lapack_int, double *, lapack_int) { DNL_SHIM_ABORT("dgesdd"); return -1; }
static inline lapack_int LAPACKE_dsyevd(int, char, char, lapack_int, double *, lapack_int, double *) { DNL_SHIM_ABORT("dsyevd"); return -1; }
static inline lapack_int LAPACKE_dgeev(int, char, char, lapack_int, double *, lapack_int, double *, double *, double *, lapack_int, double *, lapack_int) { DNL_SHIM_ABORT("dgeev"); return -1; }
#ifdef __cplusplus
}
#endif

#endif
