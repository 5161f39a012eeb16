/*
 * LAPACKE prototype shim (test infrastructure for the CPU oracle).
 *
 * The reference calls LAPACKE_dgetrf/dgetri (inverse), dgeqrf/dlacpy/dorgqr
 * (QR) and dgelqf/dorglq (LQ) in src/operator/operator_double.cpp:94-148.
 * They are mapped onto the "scipy_"-prefixed exports of scipy's OpenBLAS.
 * dsyevd is added for the oracle's HOSVD initialisation.
 */
#ifndef DT_ORACLE_LAPACKE_SHIM_H
#define DT_ORACLE_LAPACKE_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int scipy_LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double *a,
                                lapack_int lda, lapack_int *ipiv);
lapack_int scipy_LAPACKE_dgetri(int layout, lapack_int n, double *a, lapack_int lda,
                                const lapack_int *ipiv);
lapack_int scipy_LAPACKE_dgeqrf(int layout, lapack_int m, lapack_int n, double *a,
                                lapack_int lda, double *tau);
lapack_int scipy_LAPACKE_dorgqr(int layout, lapack_int m, lapack_int n, lapack_int k,
                                double *a, lapack_int lda, const double *tau);
lapack_int scipy_LAPACKE_dgelqf(int layout, lapack_int m, lapack_int n, double *a,
                                lapack_int lda, double *tau);
lapack_int scipy_LAPACKE_dorglq(int layout, lapack_int m, lapack_int n, lapack_int k,
                                double *a, lapack_int lda, const double *tau);
lapack_int scipy_LAPACKE_dlacpy(int layout, char uplo, lapack_int m, lapack_int n,
                                const double *a, lapack_int lda, double *b,
                                lapack_int ldb);
lapack_int scipy_LAPACKE_dsyevd(int layout, char jobz, char uplo, lapack_int n,
                                double *a, lapack_int lda, double *w);

#define LAPACKE_dgetrf scipy_LAPACKE_dgetrf
#define LAPACKE_dgetri scipy_LAPACKE_dgetri
#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_dorgqr scipy_LAPACKE_dorgqr
#define LAPACKE_dgelqf scipy_LAPACKE_dgelqf
#define LAPACKE_dorglq scipy_LAPACKE_dorglq
#define LAPACKE_dlacpy scipy_LAPACKE_dlacpy
#define LAPACKE_dsyevd scipy_LAPACKE_dsyevd

#ifdef __cplusplus
}
#endif
#endif
