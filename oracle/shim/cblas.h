/*
 * CBLAS prototype shim (test infrastructure for the CPU oracle).
 *
 * The reference calls cblas_dgemm / cblas_daxpy (src/operator/operator_double.cpp:168,187,208,281).
 * This image ships no CBLAS headers; scipy's bundled OpenBLAS 0.3.30 exports
 * the same routines with a "scipy_" prefix, so the reference's names are mapped
 * onto those symbols here.
 */
#ifndef DT_ORACLE_CBLAS_SHIM_H
#define DT_ORACLE_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef CBLAS_ORDER CBLAS_LAYOUT;

void scipy_cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                       int m, int n, int k, double alpha, const double *a, int lda,
                       const double *b, int ldb, double beta, double *c, int ldc);
void scipy_cblas_daxpy(int n, double alpha, const double *x, int incx, double *y,
                       int incy);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_daxpy scipy_cblas_daxpy

#ifdef __cplusplus
}
#endif
#endif
