/*
 * ORACLE (test infrastructure, never part of the product path).
 *
 * extern "C" entry points over the reference's own dense HOOI code, compiled
 * in place from the reference sources by oracle/Makefile into
 * oracle/_ref/libdiana_ref.so.  Every function here builds the reference's
 * Tensor<double> objects on a DistributionCartesianBlock({1,...,1}, 0) grid
 * (the world of size 1 that the size-1 MPI shim provides), copies the caller's
 * column-major buffers in, calls the reference routine unmodified and copies
 * the result out.
 *
 *   ref_ttm            -> Function::ttm            template/function/tensor.tpp:272-335
 *   ref_gram           -> Function::gram           template/function/tensor.tpp:18-120
 *   ref_ttt_except     -> Function::ttt_except     template/function/tensor.tpp:132-259
 *   ref_reduced_qr     -> Function::reduced_QR     template/function/matrix.tpp:86-101
 *   ref_inverse        -> Function::inverse        template/function/matrix.tpp:56-67
 *   ref_als            -> Algorithm::Tucker::ALS_  template/algorithm/tucker/hooi_als.tpp:7-34
 *   ref_hooi_als       -> Algorithm::Tucker::HOOI_ALS  hooi_als.tpp:64-123 (random init,
 *                         drawn on one thread so the initial factors are reproducible)
 *   ref_hooi_als_mt    -> the same call with every OpenMP thread the caller asks for,
 *                         the reference's normal configuration (its randn then draws
 *                         std::rand() from several threads, so the start varies)
 *   ref_hooi_harness   -> the HOOI_ALS sweep (hooi_als.tpp:94-114) composed from
 *                         Function::ttm + ALS_, with HOSVD init (Function::gram +
 *                         LAPACKE_dsyevd) and a fit-change stop rule; the
 *                         reference has neither, so the harness adds them around
 *                         its own building blocks.
 */
#include "tensor.hpp"
#include "function.hpp"
#include "algorithm.hpp"
#include "summary.hpp"

extern "C" {
#include "lapacke.h"
}

#include <omp.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

shape_t to_shape(int ndim, const int64_t *shape) {
    shape_t s;
    for (int i = 0; i < ndim; i++) s.push_back((size_t)shape[i]);
    return s;
}

DistributionCartesianBlock *unit_grid(int ndim) {
    shape_t par((size_t)ndim, 1);
    return new DistributionCartesianBlock(par, 0);
}

Tensor<double> dense_in(const double *X, const shape_t &shape) {
    Tensor<double> t(unit_grid((int)shape.size()), shape, false);
    std::memcpy(t.data(), X, t.size() * sizeof(double));
    return t;
}

Tensor<double> global_matrix_in(const double *M, size_t rows, size_t cols) {
    Tensor<double> t(new DistributionGlobal(), {rows, cols}, false);
    std::memcpy(t.data(), M, rows * cols * sizeof(double));
    return t;
}

Tensor<double> local_matrix_in(const double *M, size_t rows, size_t cols) {
    Tensor<double> t({rows, cols}, false);
    std::memcpy(t.data(), M, rows * cols * sizeof(double));
    return t;
}

void out(const Tensor<double> &t, double *dst) {
    std::memcpy(dst, t.data(), t.size() * sizeof(double));
}

/* Leading-R eigenvectors of a symmetric n x n matrix (column-major), largest
 * eigenvalue first. */
Tensor<double> leading_eigvecs(const Tensor<double> &S, size_t R) {
    const size_t n = S.shape()[0];
    std::vector<double> a(S.data(), S.data() + n * n);
    std::vector<double> w(n);
    LAPACKE_dsyevd(LAPACK_COL_MAJOR, 'V', 'U', (lapack_int)n, a.data(), (lapack_int)n,
                   w.data());
    Tensor<double> U({n, R}, false);
    for (size_t r = 0; r < R; r++) {
        const double *col = a.data() + (n - 1 - r) * n;
        std::memcpy(U.data() + r * n, col, n * sizeof(double));
    }
    return U;
}

}  // namespace

extern "C" {

int ref_ttm(const double *X, int ndim, const int64_t *shape, int mode, const double *M,
            int64_t J, double *Y) {
    shape_t s = to_shape(ndim, shape);
    auto A = dense_in(X, s);
    auto Mt = global_matrix_in(M, (size_t)J, s[(size_t)mode]);
    auto R = Function::ttm<double>(A, Mt, (size_t)mode);
    out(R, Y);
    return 0;
}

int ref_gram(const double *X, int ndim, const int64_t *shape, int mode, double *G) {
    auto A = dense_in(X, to_shape(ndim, shape));
    auto R = Function::gram<double>(A, (size_t)mode);
    out(R, G);
    return 0;
}

int ref_ttt_except(const double *A, const int64_t *shapeA, const double *B,
                   const int64_t *shapeB, int ndim, int mode, double *C) {
    auto tA = dense_in(A, to_shape(ndim, shapeA));
    auto tB = dense_in(B, to_shape(ndim, shapeB));
    auto R = Function::ttt_except<double>(tA, tB, (size_t)mode);
    out(R, C);
    return 0;
}

int ref_reduced_qr(const double *A, int64_t m, int64_t n, double *Q, double *R) {
    auto tA = local_matrix_in(A, (size_t)m, (size_t)n);
    auto [q, r] = Function::reduced_QR<double>(tA);
    out(q, Q);
    if (R) out(r, R);
    return 0;
}

int ref_inverse(const double *A, int64_t n, double *Ainv) {
    auto tA = local_matrix_in(A, (size_t)n, (size_t)n);
    auto r = Function::inverse<double>(tA);
    out(r, Ainv);
    return 0;
}

double ref_fnorm(const double *X, int ndim, const int64_t *shape) {
    auto A = dense_in(X, to_shape(ndim, shape));
    return Function::fnorm<double>(A);
}

/* ALS_ inner solver on Y (the TTM-chain output) for mode n from L0 (I_n x R). */
int ref_als(const double *Y, int ndim, const int64_t *shape, int mode, const double *L0,
            int64_t R, int64_t max_iter, double *Q) {
    shape_t s = to_shape(ndim, shape);
    auto tY = dense_in(Y, s);
    auto L = local_matrix_in(L0, s[(size_t)mode], (size_t)R);
    auto q = Algorithm::Tucker::ALS_<double>(tY, (size_t)mode, L, (size_t)max_iter);
    out(q, Q);
    return 0;
}

/* The reference's HOOI_ALS, unmodified: random Gaussian + QR initialisation
 * drawn from std::rand after srand(seed), max_iter full sweeps.  G receives the
 * core (prod R), U[n] the I_n x R_n factors. */
int ref_hooi_als(const double *X, int ndim, const int64_t *shape, const int64_t *ranks,
                 int64_t max_iter, unsigned seed, double *G, double **U, double *g_norm,
                 double *x_norm) {
    shape_t s = to_shape(ndim, shape);
    shape_t R = to_shape(ndim, ranks);
    auto A = dense_in(X, s);
    /* Operator<double>::randn draws std::rand() inside an OpenMP loop
     * (operator_double.cpp:66-72); one thread keeps the draw order, and so
     * the initial factors, reproducible. */
    const int threads = omp_get_max_threads();
    omp_set_num_threads(1);
    std::srand(seed);
    auto [core, factors] = Algorithm::Tucker::HOOI_ALS<double>(A, R, (size_t)max_iter);
    omp_set_num_threads(threads);
    if (G) out(core, G);
    for (int n = 0; n < ndim; n++)
        if (U && U[n]) out(factors[(size_t)n], U[n]);
    if (g_norm) *g_norm = Function::fnorm<double>(core);
    if (x_norm) *x_norm = Function::fnorm<double>(A);
    return 0;
}

/* The stock HOOI_ALS call on `threads` OpenMP threads (<= 0: all of them);
 * OpenBLAS keeps its own thread pool.  This is how the reference runs in
 * production, timed as the CPU baseline. */
int ref_hooi_als_mt(const double *X, int ndim, const int64_t *shape, const int64_t *ranks,
                    int64_t max_iter, unsigned seed, int threads, double *g_norm,
                    double *x_norm) {
    shape_t s = to_shape(ndim, shape);
    shape_t R = to_shape(ndim, ranks);
    auto A = dense_in(X, s);
    const int saved = omp_get_max_threads();
    omp_set_num_threads(threads > 0 ? threads : omp_get_num_procs());
    std::srand(seed);
    auto [core, factors] = Algorithm::Tucker::HOOI_ALS<double>(A, R, (size_t)max_iter);
    if (g_norm) *g_norm = Function::fnorm<double>(core);
    if (x_norm) *x_norm = Function::fnorm<double>(A);
    omp_set_num_threads(saved);
    return 0;
}

/* HOOI sweep of hooi_als.tpp:94-114 built from the reference's Function::ttm and
 * ALS_, with HOSVD initialisation (init_hosvd != 0; else the caller's U_init)
 * and the stop rule |res_k - res_{k-1}| < tol after at least one sweep.  The
 * residual is sqrt(1 - ||G||^2/||A||^2) as printed by hooi_als.tpp:112-114.
 * Returns the number of sweeps run; res_hist (length max_iter) gets each
 * sweep's residual. */
int ref_hooi_harness(const double *X, int ndim, const int64_t *shape, const int64_t *ranks,
                     int64_t max_iter, double tol, int init_hosvd, double *const *U_init,
                     double *G, double **U, double *res_hist) {
    shape_t s = to_shape(ndim, shape);
    shape_t R = to_shape(ndim, ranks);
    const size_t N = s.size();
    auto A = dense_in(X, s);
    std::vector<Tensor<double>> Uf;
    for (size_t n = 0; n < N; n++) {
        if (init_hosvd) {
            auto S = Function::gram<double>(A, n);
            Uf.push_back(leading_eigvecs(S, R[n]));
        } else {
            Uf.push_back(local_matrix_in(U_init[n], s[n], R[n]));
        }
    }
    const double a_norm = Function::fnorm<double>(A);
    double prev = -1.0;
    int sweeps = 0;
    Tensor<double> Gt;
    for (int64_t iter = 0; iter < max_iter; iter++) {
        for (size_t n = 0; n < N; n++) {
            auto Y = A.copy();
            for (size_t i = 0; i < N; i++) {
                if (i == n) continue;
                auto Ut = Function::transpose<double>(Uf[i]);
                Y = Function::ttm<double>(Y, Ut, i);
            }
            Uf[n] = Algorithm::Tucker::ALS_(Y, n, Uf[n]);
        }
        Gt = A.copy();
        for (size_t n = 0; n < N; n++) {
            auto Ut = Function::transpose<double>(Uf[n]);
            Gt = Function::ttm<double>(Gt, Ut, n);
        }
        const double g_norm = Function::fnorm<double>(Gt);
        const double res = std::sqrt(1 - (g_norm * g_norm) / (a_norm * a_norm));
        if (res_hist) res_hist[iter] = res;
        sweeps = (int)iter + 1;
        if (prev >= 0.0 && std::fabs(res - prev) < tol) break;
        prev = res;
    }
    if (G) out(Gt, G);
    for (size_t n = 0; n < N; n++)
        if (U && U[n]) out(Uf[n], U[n]);
    return sweeps;
}

// read_data<double> (src/read_data.cpp:36-129) on a .tns file: first call
// parses and returns ndim / nnz; the second copies dims, the 0-based indices
// (ndim x nnz, mode-major) and the values, then frees the buffers.
static data_buffer<double> g_tns;

int ref_read_tns(const char *path, int64_t *ndim, int64_t *nnz) {
    read_data<double>(const_cast<char *>(path), &g_tns);
    *ndim = (int64_t)g_tns.ndim;
    *nnz = (int64_t)g_tns.nnz;
    return 0;
}

int ref_read_tns_copy(int64_t *dims, int64_t *idx, double *vals) {
    const size_t nd = g_tns.ndim, nz = g_tns.nnz;
    for (size_t m = 0; m < nd; m++) {
        dims[m] = (int64_t)g_tns.dims[m];
        for (size_t e = 0; e < nz; e++) idx[m * nz + e] = (int64_t)g_tns.index_lists[m][e];
        free(g_tns.index_lists[m]);
    }
    for (size_t e = 0; e < nz; e++) vals[e] = g_tns.vals[e];
    free(g_tns.index_lists);
    free(g_tns.vals);
    free(g_tns.dims);
    g_tns = data_buffer<double>();
    return 0;
}

}  // extern "C"
