// Internal launchers shared by the operator entry points and the HOOI drivers.
// All pointers are device pointers; work is queued on ctx->stream.
#pragma once

#include "dt_core.cuh"

namespace dt {

// ---- dense FP64 (CUDA-core) kernels: dt_dense.cu --------------------------
// A dense tensor seen around mode n is a 3-way array X[l, i, b] with
// l < L = prod_{m<n} I_m (unit stride), i < I = I_n (stride L) and
// b < B = prod_{m>n} I_m (stride L*I).

// Y[l, j, b] = sum_i M(j, i) * X[l, i, b]   (Y is L x J x B), with
// M(j, i) = M[j*msj + i*msi]: (msj, msi) = (1, J) for a J x I col-major M,
// (I, 1) for the transpose of an I x J col-major factor U.
template <class TX>
void ttm_f64(dt_ctx *ctx, const TX *X, int64_t L, int64_t I, int64_t B, const double *M,
             int64_t msj, int64_t msi, int64_t J, double *Y);

// C[i, j] = sum_{l,b} A[l, i, b] * Bt[l, j, b]   (C is IA x IB col-major).
void ttt_f64(dt_ctx *ctx, const double *A, const double *Bt, int64_t L, int64_t IA,
             int64_t IB, int64_t B, double *C);

// ttt_f64 with the split-K partial tiles in caller-provided device scratch of
// scratch_doubles doubles (>= IA * IB); allocates nothing.
void ttt_f64_scratch(dt_ctx *ctx, const double *A, const double *Bt, int64_t L, int64_t IA,
                     int64_t IB, int64_t B, double *C, double *scratch, int64_t scratch_doubles);

// out[0] = sum x[e]^2 (deterministic two-stage reduction).  dtype DT_F64/DT_F32.
void sumsq(dt_ctx *ctx, const void *x, int dtype, int64_t n, double *out);

// y[e] = (double) x[e]
void f32_to_f64(dt_ctx *ctx, const float *x, int64_t n, double *y);

// Column-major C(m x n) = op(A) op(B) (FP64, small and medium sizes).
void gemm_f64(dt_ctx *ctx, int transA, int transB, int64_t m, int64_t n, int64_t k,
              const double *A, int64_t lda, const double *B, int64_t ldb, double *C,
              int64_t ldc, double beta);

// ---- small dense linear algebra: dt_linalg.cu -----------------------------
// Householder QR (LAPACK dgeqrf/dorgqr reflector convention) of the m x n
// col-major A (m >= n).  Q (m x n) and optionally R (n x n).  work >= m*n+n.
void householder_qr(dt_ctx *ctx, const double *A, int64_t m, int64_t n, double *Q,
                    double *R, double *work);

// Householder QR of `count` matrices in one launch (one CTA each): Q[b] (m[b]
// x n[b]) from A[b].  Host arrays of device pointers.
void householder_qr_batch(dt_ctx *ctx, int count, const double *const *A, double *const *Q,
                          const int64_t *m, const int64_t *n);

// Orthonormal bases Q[b] of span(A[b]) for a batch (CholeskyQR2 on the FP64
// tensor-core path, Householder on breakdown or for large matrices).
void orth_batch(dt_ctx *ctx, int count, const double *const *A, double *const *Q,
                const int64_t *m, const int64_t *n);

// Orthonormal basis of span(S^iters L) for the n x n symmetric S and the n x r
// col-major L (in place), one CTA; CholeskyQR2 per step with a Householder
// fallback.  work >= 3*n*r + r.  Sets *flag bit 2 when a fallback ran.
void subspace_iter(dt_ctx *ctx, const double *S, int64_t n, double *L, int64_t r, int iters,
                   double *work, int *flag);

// LU inverse with partial pivoting (one CTA).  *flag = 1 on a zero pivot.
void lu_inverse(dt_ctx *ctx, const double *A, int64_t n, double *Ainv, double *work,
                int *flag);

// Modified Gram-Schmidt over the len1 rows of a len1 x len2 col-major A.
void orth2_rows(dt_ctx *ctx, double *A, int64_t len1, int64_t len2);

}  // namespace dt
