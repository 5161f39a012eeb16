// Host-side interface of the tensor-core kernels (dt_tc.cu).
#pragma once

#include <cuda_bf16.h>

#include "dt_core.cuh"

namespace dt {

// Output addressing of a TTM epilogue: element (row (l', b'), column j) goes
// to  sum_d digit_d(l') * sl[d] + sum_d digit_d(b') * sb[d] + j * jstride,
// where l' and b' are split into mixed-radix digits (lowest first) of sizes
// dl[] / db[].  The folded layout Y[l, j, b] is nl = nb = 1, sl = {1},
// sb = {L*J}, jstride = L; a K-major unfolding Y_(n) uses one digit per mode.
struct OutMap {
    int nl = 0, nb = 0;
    int64_t dl[8] = {}, sl[8] = {};
    int64_t db[8] = {}, sb[8] = {};
    int64_t jstride = 0;
};

struct TcTtmArgs {
    int kmajor;  // 1: contracted index contiguous (L == 1); 0: output rows contiguous
    int64_t L, I, B;
    int J, Jpad, Npad;
    int split;  // A = hi + lo, B = [U_hi | U_lo]
    int kchunks, ksteps;
    int kbox_rows, kboxes;  // MN-major: k rows per TMA box, boxes per half-tile
    int64_t nmb, ntiles;
    int stages;
    uint32_t tx_bytes;
    int tmem_cols;
    const double *U;  // I x J col-major
    __nv_bfloat16 *out_hi, *out_lo;
    float *out_f32;
    OutMap om;
    int *err;
};

struct TcGramArgs {
    int split;
    int Ipad, N;
    int64_t kchunks_total;
    int chunks_per_cta;
    uint32_t chunk_bytes, tx_bytes;
    int tmem_cols;
    float *part;
    int *err;
};

bool tc_ttm_supported(int64_t L, int64_t I, int64_t B, int64_t J);
// Y = X x_n U^T on the tensor cores, X seen as [l, i, b] with strides
// (1, L, L*I).  Xl may be NULL (X in BF16 only); out_lo may be NULL; with
// out_f32 non-NULL the result is written in FP32 instead of BF16.  U is split
// into hi + lo when X is (or usplit > 0 with a BF16-only X: one MMA of
// X_hi [U_hi | U_lo]); usplit < 0 follows X.
void tc_ttm(dt_ctx *ctx, const __nv_bfloat16 *Xh, const __nv_bfloat16 *Xl, int64_t L, int64_t I,
            int64_t B, const double *U, int64_t J, const OutMap &om, __nv_bfloat16 *out_hi,
            __nv_bfloat16 *out_lo, float *out_f32, int *err, int usplit = -1);

bool tc_gram_supported(int64_t I, int64_t K);
// S (I x I, FP64) = Y Y^T for the K-major BF16 Y (I rows of K); with Yl the
// hi/lo cross terms are added.
// `scratch` (tc_gram_scratch_bytes) holds the split-K partial tiles; NULL
// takes a stream-ordered allocation.
void tc_gram(dt_ctx *ctx, const __nv_bfloat16 *Yh, const __nv_bfloat16 *Yl, int64_t I, int64_t K,
             double *S, int *err, void *scratch = nullptr);
size_t tc_gram_scratch_bytes(int64_t I, int64_t K, bool split);

// The same over an FP32 upload in flight: each chunk is rounded as soon as it
// has landed.
void split_f32_chunks(dt_ctx *ctx, const ChunkedUpload &up, __nv_bfloat16 *hi,
                      __nv_bfloat16 *lo, double *sumsq_out);
void split_f32(dt_ctx *ctx, const float *x, int64_t n, __nv_bfloat16 *hi, __nv_bfloat16 *lo,
               double *sumsq_out);

// G[k + K*r] = sum_i Y[i*K + k] U[i + I*r] (FP64 accumulate), ||G||^2 -> g2_out.
// `scratch` (core_rows_scratch_bytes) holds the per-block partial sums; NULL
// takes a stream-ordered allocation.
void core_rows(dt_ctx *ctx, const __nv_bfloat16 *Yh, const __nv_bfloat16 *Yl, int64_t I, int64_t K,
               const double *U, int64_t R, double *G, double *g2_out, void *scratch = nullptr);
size_t core_rows_scratch_bytes(int64_t K);

}  // namespace dt
