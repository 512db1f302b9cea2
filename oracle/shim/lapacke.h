/*
 * oracle/shim/lapacke.h -- TEST INFRASTRUCTURE ONLY (checker, never shipped).
 *
 * The single LAPACKE routine the reference calls: LAPACKE_dgesv at
 * src/math_utils.c:219 (row-major, one right-hand side). The reference passes
 * an `int *ipiv` (src/math_utils.c:189,194), so lapack_int is 32-bit here; the
 * OpenBLAS bridge converts to the ILP64 pivot array the bundled library wants.
 */
#ifndef SPIRES_ORACLE_LAPACKE_H
#define SPIRES_ORACLE_LAPACKE_H

#ifdef __cplusplus
extern "C" {
#endif

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

lapack_int LAPACKE_dgesv(int matrix_layout, lapack_int n, lapack_int nrhs,
                         double *a, lapack_int lda, lapack_int *ipiv,
                         double *b, lapack_int ldb);

#ifdef __cplusplus
}
#endif
#endif
