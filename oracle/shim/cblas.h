/*
 * oracle/shim/cblas.h -- TEST INFRASTRUCTURE ONLY (checker, never shipped).
 *
 * Minimal CBLAS interface used when the reference spires sources are compiled
 * from source for the parity oracle (oracle/_ref). Only the routines the
 * reference calls are declared:
 *   cblas_dgemv  src/reservoir.c:134,188,655,729,740  src/math_utils.c:13,48
 *   cblas_ddot   src/synapses/simple.c:63  src/reservoir.c:734
 *   cblas_dgemm  src/math_utils.c:157
 *   cblas_dscal  src/sparse.c:89  src/synapses/simple.c:71  src/reservoir.c:737,759
 *   cblas_daxpy  src/reservoir.c:275
 *   cblas_dger   src/reservoir.c:747,753
 *
 * Two implementations exist behind this header:
 *   refblas.c         -- netlib reference-BLAS summation order (bit-parity oracle)
 *   openblas_bridge.c -- forwards to the OpenBLAS build bundled with numpy
 *                        (timed CPU baseline)
 */
#ifndef SPIRES_ORACLE_CBLAS_H
#define SPIRES_ORACLE_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Standard CBLAS enumerator values (shared by every CBLAS implementation). */
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

void   cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE trans,
                   int m, int n, double alpha, const double *a, int lda,
                   const double *x, int incx, double beta, double *y, int incy);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
void   cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta,
                   enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                   const double *a, int lda, const double *b, int ldb,
                   double beta, double *c, int ldc);
void   cblas_dscal(int n, double alpha, double *x, int incx);
void   cblas_daxpy(int n, double alpha, const double *x, int incx,
                   double *y, int incy);
void   cblas_dger(enum CBLAS_ORDER order, int m, int n, double alpha,
                  const double *x, int incx, const double *y, int incy,
                  double *a, int lda);

#ifdef __cplusplus
}
#endif
#endif
