/*
 * oracle/shim/refblas.c -- TEST INFRASTRUCTURE ONLY (checker, never shipped).
 *
 * Straight-line BLAS/LAPACK routines that evaluate every sum in the order of
 * the netlib reference BLAS (LAPACK 3.x "reference BLAS" DGEMV/DDOT/DGEMM/
 * DSCAL/DAXPY/DGER and an unblocked DGETRF/DGETRS with partial pivoting).
 * Compiled with -ffp-contract=off, so every a*b+c rounds twice, exactly as the
 * reference spires sources do on x86-64 without FMA.
 *
 * Row-major CBLAS calls are mapped to the column-major Fortran routine on the
 * transposed view, exactly as the netlib CBLAS wrappers do: the order in which
 * the partial sums are formed is the one that Fortran routine uses.
 *
 * Summation orders that matter for parity with the GPU library:
 *   dgemv (row-major, no-trans)  y_i = beta*y_i (0 if beta==0), then
 *                                temp = sum_j a_ij x_j (ascending j, from +0),
 *                                y_i = y_i + alpha*temp
 *   ddot                          sequential ascending, from +0
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "cblas.h"
#include "lapacke.h"

/* Fortran DGEMV, column-major a (lda >= m), TRANS in {'N','T'}. */
static void f_dgemv(char trans, int m, int n, double alpha, const double *a,
                    int lda, const double *x, int incx, double beta, double *y,
                    int incy)
{
    int leny = (trans == 'N') ? m : n;
    int lenx = (trans == 'N') ? n : m;
    if (m == 0 || n == 0 || (alpha == 0.0 && beta == 1.0))
        return;
    int kx = incx > 0 ? 0 : -(lenx - 1) * incx;
    int ky = incy > 0 ? 0 : -(leny - 1) * incy;
    if (beta != 1.0) {
        for (int i = 0, iy = ky; i < leny; i++, iy += incy)
            y[iy] = (beta == 0.0) ? 0.0 : beta * y[iy];
    }
    if (alpha == 0.0)
        return;
    if (trans == 'N') {
        /* y := alpha*A*x + y, column sweeps */
        for (int j = 0, jx = kx; j < n; j++, jx += incx) {
            double temp = alpha * x[jx];
            for (int i = 0, iy = ky; i < m; i++, iy += incy)
                y[iy] = y[iy] + temp * a[(size_t)j * lda + i];
        }
    } else {
        /* y := alpha*A^T*x + y, one dot product per output */
        for (int j = 0, jy = ky; j < n; j++, jy += incy) {
            double temp = 0.0;
            for (int i = 0, ix = kx; i < m; i++, ix += incx)
                temp = temp + a[(size_t)j * lda + i] * x[ix];
            y[jy] = y[jy] + alpha * temp;
        }
    }
}

void cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE trans, int m,
                 int n, double alpha, const double *a, int lda, const double *x,
                 int incx, double beta, double *y, int incy)
{
    if (order == CblasColMajor)
        f_dgemv(trans == CblasNoTrans ? 'N' : 'T', m, n, alpha, a, lda, x, incx,
                beta, y, incy);
    else /* row-major A (m x n) is column-major A^T (n x m) */
        f_dgemv(trans == CblasNoTrans ? 'T' : 'N', n, m, alpha, a, lda, x, incx,
                beta, y, incy);
}

double cblas_ddot(int n, const double *x, int incx, const double *y, int incy)
{
    /* DDOT: the unrolled-by-5 form adds left to right, i.e. sequentially. */
    double s = 0.0;
    if (n <= 0)
        return s;
    int ix = incx > 0 ? 0 : -(n - 1) * incx;
    int iy = incy > 0 ? 0 : -(n - 1) * incy;
    for (int i = 0; i < n; i++, ix += incx, iy += incy)
        s = s + x[ix] * y[iy];
    return s;
}

/* Fortran DGEMM, no-trans/no-trans only (the only form the reference uses). */
static void f_dgemm_nn(int m, int n, int k, double alpha, const double *a,
                       int lda, const double *b, int ldb, double beta,
                       double *c, int ldc)
{
    for (int j = 0; j < n; j++) {
        double *cj = c + (size_t)j * ldc;
        if (beta == 0.0) {
            for (int i = 0; i < m; i++)
                cj[i] = 0.0;
        } else if (beta != 1.0) {
            for (int i = 0; i < m; i++)
                cj[i] = beta * cj[i];
        }
        for (int l = 0; l < k; l++) {
            double temp = alpha * b[(size_t)j * ldb + l];
            const double *al = a + (size_t)l * lda;
            for (int i = 0; i < m; i++)
                cj[i] = cj[i] + temp * al[i];
        }
    }
}

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb,
                 double beta, double *c, int ldc)
{
    if (ta != CblasNoTrans || tb != CblasNoTrans)
        abort(); /* not used by the reference */
    if (order == CblasColMajor)
        f_dgemm_nn(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    else /* C^T = B^T A^T in column-major terms */
        f_dgemm_nn(n, m, k, alpha, b, ldb, a, lda, beta, c, ldc);
}

void cblas_dscal(int n, double alpha, double *x, int incx)
{
    if (n <= 0 || incx <= 0)
        return;
    for (int i = 0; i < n; i++)
        x[(size_t)i * incx] = alpha * x[(size_t)i * incx];
}

void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y,
                 int incy)
{
    if (n <= 0 || alpha == 0.0)
        return;
    int ix = incx > 0 ? 0 : -(n - 1) * incx;
    int iy = incy > 0 ? 0 : -(n - 1) * incy;
    for (int i = 0; i < n; i++, ix += incx, iy += incy)
        y[iy] = y[iy] + alpha * x[ix];
}

/* Fortran DGER: A := alpha*x*y^T + A, column-major. */
static void f_dger(int m, int n, double alpha, const double *x, int incx,
                   const double *y, int incy, double *a, int lda)
{
    if (m == 0 || n == 0 || alpha == 0.0)
        return;
    int jy = incy > 0 ? 0 : -(n - 1) * incy;
    int kx = incx > 0 ? 0 : -(m - 1) * incx;
    for (int j = 0; j < n; j++, jy += incy) {
        if (y[jy] != 0.0) {
            double temp = alpha * y[jy];
            for (int i = 0, ix = kx; i < m; i++, ix += incx)
                a[(size_t)j * lda + i] = a[(size_t)j * lda + i] + x[ix] * temp;
        }
    }
}

void cblas_dger(enum CBLAS_ORDER order, int m, int n, double alpha,
                const double *x, int incx, const double *y, int incy, double *a,
                int lda)
{
    if (order == CblasColMajor)
        f_dger(m, n, alpha, x, incx, y, incy, a, lda);
    else
        f_dger(n, m, alpha, y, incy, x, incx, a, lda);
}

/*
 * LU with partial pivoting (DGETF2 order: pivot = first row of largest |a|,
 * row swap, scale the column below the pivot by 1/pivot, rank-1 update), then
 * DGETRS with one right-hand side. Row-major input is factored as given: the
 * system solved is A x = b either way.
 */
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double *a,
                         lapack_int lda, lapack_int *ipiv, double *b,
                         lapack_int ldb)
{
    if (n < 0 || nrhs < 0)
        return -1;
    /* element (i,j) of the matrix being factored */
#define A_(i, j) (*(layout == LAPACK_ROW_MAJOR ? &a[(size_t)(i) * lda + (j)] \
                                               : &a[(size_t)(j) * lda + (i)]))
#define B_(i, r) (*(layout == LAPACK_ROW_MAJOR ? &b[(size_t)(i) * ldb + (r)] \
                                               : &b[(size_t)(r) * ldb + (i)]))
    lapack_int info = 0;
    for (int j = 0; j < n; j++) {
        int p = j;
        double best = fabs(A_(j, j));
        for (int i = j + 1; i < n; i++) {
            double v = fabs(A_(i, j));
            if (v > best) {
                best = v;
                p = i;
            }
        }
        ipiv[j] = p + 1;
        if (A_(p, j) != 0.0) {
            if (p != j) {
                for (int c = 0; c < n; c++) {
                    double t = A_(j, c);
                    A_(j, c) = A_(p, c);
                    A_(p, c) = t;
                }
            }
            double rp = 1.0 / A_(j, j);
            for (int i = j + 1; i < n; i++)
                A_(i, j) = rp * A_(i, j);
        } else if (info == 0) {
            info = j + 1;
        }
        for (int c = j + 1; c < n; c++) {
            double t = A_(j, c);
            if (t != 0.0)
                for (int i = j + 1; i < n; i++)
                    A_(i, c) = A_(i, c) + A_(i, j) * (-t);
        }
    }
    if (info != 0)
        return info;
    for (int r = 0; r < nrhs; r++) {
        for (int j = 0; j < n; j++) {
            int p = ipiv[j] - 1;
            if (p != j) {
                double t = B_(j, r);
                B_(j, r) = B_(p, r);
                B_(p, r) = t;
            }
        }
        for (int j = 0; j < n; j++) { /* L y = b, unit diagonal */
            double t = B_(j, r);
            if (t != 0.0)
                for (int i = j + 1; i < n; i++)
                    B_(i, r) = B_(i, r) - t * A_(i, j);
        }
        for (int j = n - 1; j >= 0; j--) { /* U x = y */
            if (B_(j, r) != 0.0) {
                B_(j, r) = B_(j, r) / A_(j, j);
                double t = B_(j, r);
                for (int i = 0; i < j; i++)
                    B_(i, r) = B_(i, r) - t * A_(i, j);
            }
        }
    }
#undef A_
#undef B_
    return 0;
}
