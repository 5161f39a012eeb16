/*
 * ORACLE (test infrastructure, never part of the product path): a plain-C
 * restatement of the reference's sparse Tucker hot path.  The reference's
 * sparse sources do not compile as shipped (private members used from
 * Sp_HOOI_ALS, a misspelt slice_satrt, the missing v_index_buffer), so this
 * file restates the intended arithmetic:
 *
 *   orc_sp_fnorm       template/function/sp_tensor.tpp:6-14
 *   orc_sp_ttmc_rows   add_outer_product_all, sp_tensor.tpp:367-417: for every
 *                      mode-n row i, Y(i,:) = sum_{nnz with i_n=i} v * (x)_{m!=n}
 *                      U_m(i_m,:), the lowest non-n mode varying fastest.  The
 *                      reference's stride bug (sp_tensor.tpp:299 pushes R_n as
 *                      every stride) coincides with this when all R_m are equal.
 *   orc_sp_ttmc_mTR    sp_tensor.tpp:236-286, intended form L = Y_(n)^T U_n
 *                      (the shipped loop indexes R by nonzero number instead of
 *                      i_n and never resets its row accumulator).
 *   orc_sp_ttmc_mTL    sp_tensor.tpp:288-365: ret(:,i) = (Y_(n)(i,:) L)^T.
 *   orc_orth2          Operator<double>::orth2, src/operator/operator_double.cpp:248-277
 *                      (modified Gram-Schmidt over the rows of an R x I matrix).
 *   orc_sp_hooi        Sp_HOOI_ALS / Sp_TTMC_ALS_, template/algorithm/sp_tucker/
 *                      sp_hooi_als.tpp:48-118: per mode L = Y_(n)^T U_n,
 *                      U_n <- orth2(Y_(n) L); core G = mTR(N-1) after the sweeps.
 *   orc_sp_ttmc_dense  Function::ttmc(SpTensor, M, idx, ...), sp_tensor.tpp:16-192,
 *                      at world size 1 (one rank: the whole output is the local
 *                      block and the ring has one step): every nonzero, in input
 *                      order, is added by the recursion of add_outer_product
 *                      (sp_tensor.tpp:419-450), from the highest mode down; a
 *                      contracted mode m loops over the J_m entries of
 *                      M_m(:, i_m) (M_m J_m x I_m column-major), a kept mode jumps
 *                      to its index.  The output is column-major.
 *
 * Factors are passed TRANSPOSED as in the reference (sp_hooi_als.tpp:80):
 * Ut[m] is R_m x I_m column-major, so factor row i is Ut[m] + i*R_m.
 * Nonzero indices are int64, 0-based.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXD 8

/* Counting sort of the nonzeros by their mode-n index: pos has I_n+1 entries,
 * perm lists nonzero ids row by row in input order (stable). */
static void build_rows(int64_t nnz, const int64_t *idx_n, int64_t I_n, int64_t *pos,
                       int64_t *perm) {
    memset(pos, 0, (size_t)(I_n + 1) * sizeof(int64_t));
    for (int64_t e = 0; e < nnz; e++) pos[idx_n[e] + 1]++;
    for (int64_t i = 0; i < I_n; i++) pos[i + 1] += pos[i];
    int64_t *fill = (int64_t *)malloc((size_t)I_n * sizeof(int64_t));
    memcpy(fill, pos, (size_t)I_n * sizeof(int64_t));
    for (int64_t e = 0; e < nnz; e++) perm[fill[idx_n[e]]++] = e;
    free(fill);
}

double orc_sp_fnorm(int64_t nnz, const double *vals) {
    double s = 0.0;
    for (int64_t e = 0; e < nnz; e++) s += vals[e] * vals[e];
    return sqrt(s);
}

/* Accumulates v * kron_{m != n} U_m(i_m, :) into row (length P), lowest non-n
 * mode fastest. */
static void add_kron(double *row, int ndim, int mode, const int64_t *const *idx,
                     int64_t e, double v, const double *const *Ut, const int64_t *R) {
    int modes[MAXD];
    int k = 0;
    for (int m = 0; m < ndim; m++)
        if (m != mode) modes[k++] = m;
    /* Iterate the Kronecker index space with an odometer. */
    int64_t cnt[MAXD] = {0};
    const double *vec[MAXD];
    int64_t len[MAXD];
    int64_t P = 1;
    for (int d = 0; d < k; d++) {
        vec[d] = Ut[modes[d]] + idx[modes[d]][e] * R[modes[d]];
        len[d] = R[modes[d]];
        P *= len[d];
    }
    if (k == 0) {
        row[0] += v;
        return;
    }
    /* Precompute the product of the slow factors and sweep the fastest one. */
    const int64_t r0 = len[0];
    for (int64_t base = 0; base < P; base += r0) {
        double w = v;
        for (int d = 1; d < k; d++) w *= vec[d][cnt[d]];
        double *dst = row + base;
        for (int64_t t = 0; t < r0; t++) dst[t] += w * vec[0][t];
        for (int d = 1; d < k; d++) {
            if (++cnt[d] < len[d]) break;
            cnt[d] = 0;
        }
    }
}

static int64_t kron_len(int ndim, int mode, const int64_t *R) {
    int64_t P = 1;
    for (int m = 0; m < ndim; m++)
        if (m != mode) P *= R[m];
    return P;
}

/* Y rows for all mode-n rows: Y is I_n x P row-major (row i at Y + i*P). */
int orc_sp_ttmc_rows(int64_t nnz, int ndim, const int64_t *const *idx, const double *vals,
                     const int64_t *shape, const double *const *Ut, const int64_t *R,
                     int mode, double *Y) {
    const int64_t I_n = shape[mode];
    const int64_t P = kron_len(ndim, mode, R);
    int64_t *pos = (int64_t *)malloc((size_t)(I_n + 1) * sizeof(int64_t));
    int64_t *perm = (int64_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int64_t));
    build_rows(nnz, idx[mode], I_n, pos, perm);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < I_n; i++) {
        double *row = Y + i * P;
        memset(row, 0, (size_t)P * sizeof(double));
        for (int64_t j = pos[i]; j < pos[i + 1]; j++) {
            const int64_t e = perm[j];
            add_kron(row, ndim, mode, idx, e, vals[e], Ut, R);
        }
    }
    free(pos);
    free(perm);
    return 0;
}

/* L (P x R_n, column-major) = Y_(n)^T U_n. */
int orc_sp_ttmc_mTR(int64_t nnz, int ndim, const int64_t *const *idx, const double *vals,
                    const int64_t *shape, const double *const *Ut, const int64_t *R, int mode,
                    double *L) {
    const int64_t I_n = shape[mode];
    const int64_t P = kron_len(ndim, mode, R);
    const int64_t Rn = R[mode];
    int64_t *pos = (int64_t *)malloc((size_t)(I_n + 1) * sizeof(int64_t));
    int64_t *perm = (int64_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int64_t));
    build_rows(nnz, idx[mode], I_n, pos, perm);
    memset(L, 0, (size_t)(P * Rn) * sizeof(double));
#pragma omp parallel
    {
        double *row = (double *)malloc((size_t)P * sizeof(double));
        double *acc = (double *)calloc((size_t)(P * Rn), sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < I_n; i++) {
            if (pos[i] == pos[i + 1]) continue;
            memset(row, 0, (size_t)P * sizeof(double));
            for (int64_t j = pos[i]; j < pos[i + 1]; j++) {
                const int64_t e = perm[j];
                add_kron(row, ndim, mode, idx, e, vals[e], Ut, R);
            }
            const double *u = Ut[mode] + i * Rn;
            for (int64_t k = 0; k < Rn; k++) {
                const double uk = u[k];
                double *dst = acc + k * P;
                for (int64_t p = 0; p < P; p++) dst[p] += row[p] * uk;
            }
        }
#pragma omp critical
        for (int64_t t = 0; t < P * Rn; t++) L[t] += acc[t];
        free(row);
        free(acc);
    }
    free(pos);
    free(perm);
    return 0;
}

/* ret (R_n x I_n, column-major; column i = new factor row i) = (Y_(n) L)^T. */
int orc_sp_ttmc_mTL(int64_t nnz, int ndim, const int64_t *const *idx, const double *vals,
                    const int64_t *shape, const double *const *Ut, const int64_t *R, int mode,
                    const double *L, double *ret) {
    const int64_t I_n = shape[mode];
    const int64_t P = kron_len(ndim, mode, R);
    const int64_t Rn = R[mode];
    int64_t *pos = (int64_t *)malloc((size_t)(I_n + 1) * sizeof(int64_t));
    int64_t *perm = (int64_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int64_t));
    build_rows(nnz, idx[mode], I_n, pos, perm);
#pragma omp parallel
    {
        double *row = (double *)malloc((size_t)P * sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < I_n; i++) {
            double *out = ret + i * Rn;
            for (int64_t k = 0; k < Rn; k++) out[k] = 0.0;
            if (pos[i] == pos[i + 1]) continue;
            memset(row, 0, (size_t)P * sizeof(double));
            for (int64_t j = pos[i]; j < pos[i + 1]; j++) {
                const int64_t e = perm[j];
                add_kron(row, ndim, mode, idx, e, vals[e], Ut, R);
            }
            for (int64_t k = 0; k < Rn; k++) {
                const double *lk = L + k * P;
                double s = 0.0;
                for (int64_t p = 0; p < P; p++) s += row[p] * lk[p];
                out[k] = s;
            }
        }
        free(row);
    }
    free(pos);
    free(perm);
    return 0;
}

/* One nonzero's contribution below mode `dim` (add_outer_product). */
static void outer_add(double *data, const int64_t *stride, int dim, const int *contract,
                      const double *const *M, const int64_t *J, const int64_t *index,
                      double val) {
    if (contract[dim]) {
        const double *col = M[dim] + index[dim] * J[dim];
        for (int64_t j = 0; j < J[dim]; j++) {
            if (dim == 0)
                data[j] += val * col[j];
            else
                outer_add(data + stride[dim] * j, stride, dim - 1, contract, M, J, index,
                          val * col[j]);
        }
    } else if (dim == 0) {
        data[index[0]] += val;
    } else {
        outer_add(data + stride[dim] * index[dim], stride, dim - 1, contract, M, J, index, val);
    }
}

/* Y (column-major; mode m has extent J[m] if contract[m], else shape[m]). */
int orc_sp_ttmc_dense(int64_t nnz, int ndim, const int64_t *const *idx, const double *vals,
                      const int64_t *shape, const double *const *M, const int64_t *J,
                      const int *contract, double *Y) {
    int64_t stride[MAXD], total = 1;
    for (int m = 0; m < ndim; m++) {
        stride[m] = total;
        total *= contract[m] ? J[m] : shape[m];
    }
    memset(Y, 0, (size_t)total * sizeof(double));
    int64_t index[MAXD];
    for (int64_t e = 0; e < nnz; e++) {
        for (int m = 0; m < ndim; m++) index[m] = idx[m][e];
        outer_add(Y, stride, ndim - 1, contract, M, J, index, vals[e]);
    }
    return 0;
}

/* Modified Gram-Schmidt over the len1 rows of a len1 x len2 column-major
 * matrix, exactly the loop order of Operator<double>::orth2. */
void orc_orth2(double *A, int64_t len1, int64_t len2) {
    for (int64_t i = 0; i < len1; i++) {
        for (int64_t j = 0; j < i; j++) {
            double dot = 0.0;
            for (int64_t k = 0; k < len2; k++) dot += A[k * len1 + i] * A[k * len1 + j];
            for (int64_t k = 0; k < len2; k++) A[k * len1 + i] -= A[k * len1 + j] * dot;
        }
        double norm = 0.0;
        for (int64_t k = 0; k < len2; k++) norm += A[k * len1 + i] * A[k * len1 + i];
        norm = sqrt(norm);
        for (int64_t k = 0; k < len2; k++) A[k * len1 + i] /= norm;
    }
}

/* Sparse HOOI power sweeps.  Ut[m] (R_m x I_m) holds the initial factors on
 * entry and the final ones on exit.  G (P_{N-1} x R_{N-1}, i.e. the core in
 * column-major order) and the residual sqrt(1-||G||^2/||A||^2) are returned. */
int orc_sp_hooi(int64_t nnz, int ndim, const int64_t *const *idx, const double *vals,
                const int64_t *shape, const int64_t *R, int64_t max_iter, double **Ut,
                double *G, double *residual) {
    const double a_norm = orc_sp_fnorm(nnz, vals);
    for (int64_t it = 0; it < max_iter; it++) {
        for (int n = 0; n < ndim; n++) {
            const int64_t P = kron_len(ndim, n, R);
            double *L = (double *)malloc((size_t)(P * R[n]) * sizeof(double));
            orc_sp_ttmc_mTR(nnz, ndim, idx, vals, shape, (const double *const *)Ut, R, n, L);
            orc_sp_ttmc_mTL(nnz, ndim, idx, vals, shape, (const double *const *)Ut, R, n, L,
                            Ut[n]);
            orc_orth2(Ut[n], R[n], shape[n]);
            free(L);
        }
    }
    const int last = ndim - 1;
    const int64_t P = kron_len(ndim, last, R);
    double *L = G ? G : (double *)malloc((size_t)(P * R[last]) * sizeof(double));
    orc_sp_ttmc_mTR(nnz, ndim, idx, vals, shape, (const double *const *)Ut, R, last, L);
    double g2 = 0.0;
    for (int64_t t = 0; t < P * R[last]; t++) g2 += L[t] * L[t];
    if (residual) *residual = sqrt(1.0 - g2 / (a_norm * a_norm));
    if (!G) free(L);
    return 0;
}
