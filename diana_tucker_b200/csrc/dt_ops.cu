// extern "C" operator-level entry points (the Function:: / Operator<double>
// seam of the reference) over the FP64 kernels.
#include "dt_kernels.cuh"

using namespace dt;

namespace {

struct ModeView {
    int64_t L, I, B;
};

ModeView around(int ndim, const int64_t *shape, int mode) {
    ModeView v{1, shape[mode], 1};
    for (int m = 0; m < mode; m++) v.L *= shape[m];
    for (int m = mode + 1; m < ndim; m++) v.B *= shape[m];
    return v;
}

void read_flag(dt_ctx *ctx, const DevMem &flag, int *h) {
    DT_CUDA(cudaMemcpyAsync(h, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace

extern "C" {

int dt_ttm_f64(dt_ctx *ctx, const double *X, int ndim, const int64_t *shape, int mode,
               const double *M, int64_t J, double *Y) {
    return guard([&] {
        check_ctx(ctx);
        check_shape(ndim, shape, "dt_ttm_f64");
        DT_CHECK_ARG(mode >= 0 && mode < ndim, "dt_ttm_f64: mode %d out of range", mode);
        DT_CHECK_ARG(J >= 1, "dt_ttm_f64: J must be >= 1");
        DT_CUDA(cudaSetDevice(ctx->device));
        const ModeView v = around(ndim, shape, mode);
        const int64_t nx = v.L * v.I * v.B, ny = v.L * J * v.B;
        DevView x(ctx, X, nx * sizeof(double), true, false);
        DevView m(ctx, M, J * v.I * sizeof(double), true, false);
        DevView y(ctx, Y, ny * sizeof(double), false, true);
        SummaryScope sc(ctx, "Function::ttm()", 2.0 * nx * J, 8.0 * (nx + ny + J * v.I));
        ttm_f64<double>(ctx, x.as<double>(), v.L, v.I, v.B, m.as<double>(), 1, J, J,
                        y.as<double>());
        y.finish();
    });
}

int dt_gram_f64(dt_ctx *ctx, const double *X, int ndim, const int64_t *shape, int mode,
                double *G) {
    return guard([&] {
        check_ctx(ctx);
        check_shape(ndim, shape, "dt_gram_f64");
        DT_CHECK_ARG(mode >= 0 && mode < ndim, "dt_gram_f64: mode %d out of range", mode);
        DT_CUDA(cudaSetDevice(ctx->device));
        const ModeView v = around(ndim, shape, mode);
        DevView x(ctx, X, v.L * v.I * v.B * sizeof(double), true, false);
        DevView g(ctx, G, v.I * v.I * sizeof(double), false, true);
        SummaryScope sc(ctx, "Function::gram()", 2.0 * v.L * v.I * v.B * v.I,
                        8.0 * (v.L * v.I * v.B + v.I * v.I));
        ttt_f64(ctx, x.as<double>(), x.as<double>(), v.L, v.I, v.I, v.B, g.as<double>());
        g.finish();
    });
}

int dt_ttt_except_f64(dt_ctx *ctx, const double *A, const int64_t *shapeA, const double *B,
                      const int64_t *shapeB, int ndim, int mode, double *C) {
    return guard([&] {
        check_ctx(ctx);
        check_shape(ndim, shapeA, "dt_ttt_except_f64");
        check_shape(ndim, shapeB, "dt_ttt_except_f64");
        DT_CHECK_ARG(mode >= 0 && mode < ndim, "dt_ttt_except_f64: mode %d out of range", mode);
        for (int m = 0; m < ndim; m++)
            if (m != mode)
                DT_CHECK_ARG(shapeA[m] == shapeB[m],
                             "dt_ttt_except_f64: shapes differ in mode %d (%lld vs %lld)", m,
                             (long long)shapeA[m], (long long)shapeB[m]);
        DT_CUDA(cudaSetDevice(ctx->device));
        const ModeView va = around(ndim, shapeA, mode);
        const int64_t IB = shapeB[mode];
        DevView a(ctx, A, va.L * va.I * va.B * sizeof(double), true, false);
        DevView b(ctx, B, va.L * IB * va.B * sizeof(double), true, false);
        DevView c(ctx, C, va.I * IB * sizeof(double), false, true);
        SummaryScope sc(ctx, "Function::ttt_except()", 2.0 * va.L * va.I * IB * va.B,
                        8.0 * (va.L * (va.I + IB) * va.B + va.I * IB));
        ttt_f64(ctx, a.as<double>(), b.as<double>(), va.L, va.I, IB, va.B, c.as<double>());
        c.finish();
    });
}

int dt_fnorm_f64(dt_ctx *ctx, const double *X, int64_t n, double *out) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(n >= 0 && out, "dt_fnorm_f64: bad arguments");
        DT_CUDA(cudaSetDevice(ctx->device));
        if (n == 0) {
            *out = 0.0;
            return;
        }
        DevView x(ctx, X, n * sizeof(double), true, false);
        DevMem s(ctx, sizeof(double));
        sumsq(ctx, x.ptr(), DT_F64, n, s.as<double>());
        double h = 0.0;
        DT_CUDA(cudaMemcpyAsync(&h, s.get(), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = sqrt(h);
    });
}

int dt_matmul_f64(dt_ctx *ctx, int transA, int transB, int64_t m, int64_t n, int64_t k,
                  const double *A, const double *B, double *C) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(m >= 1 && n >= 1 && k >= 1, "dt_matmul_f64: empty operand");
        DT_CHECK_ARG((transA == 0 || transA == 1) && (transB == 0 || transB == 1),
                     "dt_matmul_f64: trans must be 0 or 1");
        DT_CHECK_ARG(!(transA && transB), "dt_matmul_f64: TT is not a reference operator");
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView a(ctx, A, m * k * sizeof(double), true, false);
        DevView b(ctx, B, k * n * sizeof(double), true, false);
        DevView c(ctx, C, m * n * sizeof(double), false, true);
        const int64_t lda = transA ? k : m;
        const int64_t ldb = transB ? n : k;
        gemm_f64(ctx, transA, transB, m, n, k, a.as<double>(), lda, b.as<double>(), ldb,
                 c.as<double>(), m, 0.0);
        c.finish();
    });
}

int dt_reduced_qr_f64(dt_ctx *ctx, const double *A, int64_t m, int64_t n, double *Q,
                      double *R) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(m >= n && n >= 1, "dt_reduced_qr_f64: need m >= n >= 1");
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView a(ctx, A, m * n * sizeof(double), true, false);
        DevView q(ctx, Q, m * n * sizeof(double), false, true);
        DevView r(ctx, R, R ? n * n * sizeof(double) : 0, false, true);
        DevMem work(ctx, (m * n + n) * sizeof(double));
        householder_qr(ctx, a.as<double>(), m, n, q.as<double>(), R ? r.as<double>() : nullptr,
                       work.as<double>());
        q.finish();
        if (R) r.finish();
    });
}

int dt_inverse_f64(dt_ctx *ctx, const double *A, int64_t n, double *Ainv) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(n >= 1, "dt_inverse_f64: empty matrix");
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView a(ctx, A, n * n * sizeof(double), true, false);
        DevView o(ctx, Ainv, n * n * sizeof(double), false, true);
        DevMem work(ctx, n * n * sizeof(double));
        DevMem flag(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), ctx->stream));
        lu_inverse(ctx, a.as<double>(), n, o.as<double>(), work.as<double>(), flag.as<int>());
        int h = 0;
        read_flag(ctx, flag, &h);
        if (h) fail(DT_ERR_NUMERIC, "dt_inverse_f64: matrix is singular");
        o.finish();
    });
}

int dt_orth2_f64(dt_ctx *ctx, double *A, int64_t len1, int64_t len2) {
    return guard([&] {
        check_ctx(ctx);
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView a(ctx, A, len1 * len2 * sizeof(double), true, true);
        orth2_rows(ctx, a.as<double>(), len1, len2);
        a.finish();
    });
}

int dt_als_f64(dt_ctx *ctx, const double *Y, int ndim, const int64_t *shape, int mode,
               const double *L0, int64_t R, int iters, double *Q) {
    return guard([&] {
        check_ctx(ctx);
        check_shape(ndim, shape, "dt_als_f64");
        DT_CHECK_ARG(mode >= 0 && mode < ndim, "dt_als_f64: mode %d out of range", mode);
        DT_CHECK_ARG(R >= 1 && R <= shape[mode], "dt_als_f64: need 1 <= R <= I_n");
        DT_CHECK_ARG(iters >= 1, "dt_als_f64: iters must be >= 1");
        DT_CUDA(cudaSetDevice(ctx->device));
        const ModeView v = around(ndim, shape, mode);
        DevView y(ctx, Y, v.L * v.I * v.B * sizeof(double), true, false);
        DevView l0(ctx, L0, v.I * R * sizeof(double), true, false);
        DevView q(ctx, Q, v.I * R * sizeof(double), false, true);
        DevMem S(ctx, v.I * v.I * sizeof(double));
        DevMem work(ctx, (3 * v.I * R + R) * sizeof(double));
        DevMem flag(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), ctx->stream));
        SummaryScope sc(ctx, "Algorithm::Tucker::ALS_()",
                        2.0 * v.L * v.I * v.B * v.I + 2.0 * iters * v.I * v.I * R,
                        8.0 * (v.L * v.I * v.B + v.I * v.I));
        ttt_f64(ctx, y.as<double>(), y.as<double>(), v.L, v.I, v.I, v.B, S.as<double>());
        DT_CUDA(cudaMemcpyAsync(q.ptr(), l0.ptr(), v.I * R * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        subspace_iter(ctx, S.as<double>(), v.I, q.as<double>(), R, iters, work.as<double>(),
                      flag.as<int>());
        q.finish();
    });
}

}  // extern "C"
