/*
 * oracle/shim/openblas_bridge.c -- TEST INFRASTRUCTURE ONLY (timed CPU baseline).
 *
 * Forwards the CBLAS/LAPACKE calls of the reference sources to the ILP64
 * OpenBLAS 0.3.x build that numpy bundles (exported with a `scipy_` prefix and
 * a `64_` suffix). Integers widen to 64 bits; the 32-bit pivot array the
 * reference hands to LAPACKE_dgesv (src/math_utils.c:189,219) is converted.
 * This variant is only used to time the reference on the host cores; the
 * bit-parity oracle uses refblas.c instead.
 */
#include <stdint.h>
#include <stdlib.h>
#include "cblas.h"
#include "lapacke.h"

typedef int64_t bi;

extern void scipy_cblas_dgemv64_(int, int, bi, bi, double, const double *, bi,
                                 const double *, bi, double, double *, bi);
extern double scipy_cblas_ddot64_(bi, const double *, bi, const double *, bi);
extern void scipy_cblas_dgemm64_(int, int, int, bi, bi, bi, double,
                                 const double *, bi, const double *, bi, double,
                                 double *, bi);
extern void scipy_cblas_dscal64_(bi, double, double *, bi);
extern void scipy_cblas_daxpy64_(bi, double, const double *, bi, double *, bi);
extern void scipy_cblas_dger64_(int, bi, bi, double, const double *, bi,
                                const double *, bi, double *, bi);
extern bi scipy_LAPACKE_dgesv64_(int, bi, bi, double *, bi, bi *, double *, bi);

void cblas_dgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int m, int n,
                 double alpha, const double *a, int lda, const double *x,
                 int incx, double beta, double *y, int incy)
{
    scipy_cblas_dgemv64_(o, t, m, n, alpha, a, lda, x, incx, beta, y, incy);
}

double cblas_ddot(int n, const double *x, int incx, const double *y, int incy)
{
    return scipy_cblas_ddot64_(n, x, incx, y, incy);
}

void cblas_dgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb,
                 double beta, double *c, int ldc)
{
    scipy_cblas_dgemm64_(o, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c,
                         ldc);
}

void cblas_dscal(int n, double alpha, double *x, int incx)
{
    scipy_cblas_dscal64_(n, alpha, x, incx);
}

void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y,
                 int incy)
{
    scipy_cblas_daxpy64_(n, alpha, x, incx, y, incy);
}

void cblas_dger(enum CBLAS_ORDER o, int m, int n, double alpha,
                const double *x, int incx, const double *y, int incy, double *a,
                int lda)
{
    scipy_cblas_dger64_(o, m, n, alpha, x, incx, y, incy, a, lda);
}

lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double *a,
                         lapack_int lda, lapack_int *ipiv, double *b,
                         lapack_int ldb)
{
    bi *piv = malloc((size_t)(n > 0 ? n : 1) * sizeof(bi));
    if (!piv)
        return -1;
    bi info = scipy_LAPACKE_dgesv64_(layout, n, nrhs, a, lda, piv, b, ldb);
    for (lapack_int i = 0; i < n; i++)
        ipiv[i] = (lapack_int)piv[i];
    free(piv);
    return (lapack_int)info;
}
