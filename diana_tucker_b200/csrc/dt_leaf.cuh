// The leaf Grams of a pair node of the dense HOOI tree, straight from the
// pair's intermediate (dt_leaf.cu).
#pragma once

#include <cuda_bf16.h>

#include "dt_core.cuh"

namespace dt {

bool pair_gram_supported(int64_t np, int64_t nq, int64_t R);
// Doubles of partial-Gram scratch pair_gram needs at most.
size_t pair_gram_scratch_doubles(int64_t np, int64_t nq, int64_t nc);

// S (FP64, col-major) = Y_(p) Y_(p)^T (side 0) or Y_(q) Y_(q)^T (side 1) of
// the pair intermediate T (BF16 hi + optional lo): element (i, j, c) at
// i*sp + j*sq + (c % clo) + (c / clo)*chs, i < np, j < nq, c < nc; U is the
// factor of the contracted mode (q for side 0, p for side 1), n x R col-major.
void pair_gram(dt_ctx *ctx, const __nv_bfloat16 *Th, const __nv_bfloat16 *Tl, int64_t np,
               int64_t nq, int64_t sp, int64_t sq, int64_t clo, int64_t chs, int64_t nc, int side,
               const double *U, int64_t R, double *part, size_t part_doubles, double *S);

// L (n x R col-major, in place) <- orth(S^iters L) for a symmetric n x n S,
// n <= 128, R <= 32, in one CTA on the FP64 tensor cores (CholeskyQR after
// every second product, CholeskyQR2 at the end; modified Gram-Schmidt and
// bit 2 of *flag on breakdown).  With g2_out: trace(L^T S L) of the result.
bool subspace_small_supported(int64_t n, int64_t R);
void subspace_small(dt_ctx *ctx, const double *S, int64_t n, double *L, int64_t R, int iters,
                    int *flag, double *g2_out);

// T (R0 x R1 x S col-major, FP64) = X x_0 U0^T x_1 U1^T for the FP32 X seen
// as I0 x I1 x S, in one pass over X on the FP64 tensor cores (dt_core_proj.cu).
bool core_slices_supported(int64_t I0, int64_t I1, int64_t R0, int64_t R1);
void core_slices_f64(dt_ctx *ctx, const float *X, int64_t I0, int64_t I1, int64_t S,
                     const double *U0, int64_t R0, const double *U1, int64_t R1, double *T);

// out[0] = trace(U^T S U) for S n x n, U n x R (FP64).
void quad_trace(dt_ctx *ctx, const double *S, int64_t n, const double *U, int64_t R, double *out);

}  // namespace dt
