// extern "C" entry points for the tensor-core operators on their own
// (mixed-precision TTM and Gram), used by the HOOI driver internally.
#include "dt_kernels.cuh"
#include "dt_tc.cuh"
#include "dt_tc_host.cuh"

using namespace dt;

namespace {

// One mbarrier that nothing arrives on: every thread's bounded wait runs out,
// records the timeout in the error word, and the kernel returns.  No copy or
// MMA is issued, so nothing is in flight when it exits.
__global__ void wait_selftest_kernel(int *err, long long limit) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    tc::mbar_wait(&bar, 0, err, limit);
}

}  // namespace

extern "C" {

int dt_selftest_wait_timeout(dt_ctx *ctx, int64_t limit_cycles) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(limit_cycles >= 0 && limit_cycles <= tc::kWaitCycles,
                     "dt_selftest_wait_timeout: limit %lld outside [0, %lld]",
                     (long long)limit_cycles, (long long)tc::kWaitCycles);
        DT_CUDA(cudaSetDevice(ctx->device));
        DevMem err(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), ctx->stream));
        DT_LAUNCH(ctx, wait_selftest_kernel, 1, 32, 0, err.as<int>(), (long long)limit_cycles);
        int h = 0;
        DT_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h) fail(DT_ERR_TIMEOUT, fmt("self-test: the bounded wait ran out after %lld cycles "
                                        "(error word %d)", (long long)limit_cycles, h));
    });
}

int dt_ttm_tc(dt_ctx *ctx, const float *X, int ndim, const int64_t *shape, int mode,
              const double *U, int64_t J, int split, float *Y) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(ndim >= 1 && ndim <= 16 && shape && X && U && Y, "dt_ttm_tc: bad arguments");
        DT_CHECK_ARG(mode >= 0 && mode < ndim, "dt_ttm_tc: mode %d out of range", mode);
        DT_CUDA(cudaSetDevice(ctx->device));
        int64_t L = 1, B = 1;
        for (int m = 0; m < mode; m++) L *= shape[m];
        for (int m = mode + 1; m < ndim; m++) B *= shape[m];
        const int64_t I = shape[mode];
        if (!tc_ttm_supported(L, I, B, J))
            fail(DT_ERR_UNSUPPORTED,
                 fmt("dt_ttm_tc: layout outside the TMA rules (L=%lld I=%lld J=%lld)",
                     (long long)L, (long long)I, (long long)J));
        const int64_t nx = L * I * B, ny = L * J * B;
        DevView x(ctx, X, nx * sizeof(float), true, false);
        DevView u(ctx, U, I * J * sizeof(double), true, false);
        DevView y(ctx, Y, ny * sizeof(float), false, true);
        DevMem xh(ctx, nx * 2), xl(ctx, split ? nx * 2 : 0), s2(ctx, sizeof(double)),
            err(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), ctx->stream));
        split_f32(ctx, x.as<float>(), nx, xh.as<__nv_bfloat16>(),
                  split ? xl.as<__nv_bfloat16>() : nullptr, s2.as<double>());
        OutMap om;
        om.nl = 1;
        om.dl[0] = L;
        om.sl[0] = 1;
        om.nb = 1;
        om.db[0] = B;
        om.sb[0] = L * J;
        om.jstride = L;
        tc_ttm(ctx, xh.as<__nv_bfloat16>(), split ? xl.as<__nv_bfloat16>() : nullptr, L, I, B,
               u.as<double>(), J, om, nullptr, nullptr, y.as<float>(), err.as<int>());
        int h = 0;
        DT_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h) fail(DT_ERR_TIMEOUT, "dt_ttm_tc: a tensor-core wait timed out");
        y.finish();
    });
}

int dt_gram_tc(dt_ctx *ctx, const float *Y, int64_t I, int64_t K, int split, double *S) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(Y && S, "dt_gram_tc: null argument");
        DT_CUDA(cudaSetDevice(ctx->device));
        if (!tc_gram_supported(I, K))
            fail(DT_ERR_UNSUPPORTED, fmt("dt_gram_tc: unsupported I=%lld K=%lld", (long long)I,
                                         (long long)K));
        DevView y(ctx, Y, I * K * sizeof(float), true, false);
        DevView s(ctx, S, I * I * sizeof(double), false, true);
        DevMem yh(ctx, I * K * 2), yl(ctx, split ? I * K * 2 : 0), s2(ctx, sizeof(double)),
            err(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), ctx->stream));
        split_f32(ctx, y.as<float>(), I * K, yh.as<__nv_bfloat16>(),
                  split ? yl.as<__nv_bfloat16>() : nullptr, s2.as<double>());
        tc_gram(ctx, yh.as<__nv_bfloat16>(), split ? yl.as<__nv_bfloat16>() : nullptr, I, K,
                s.as<double>(), err.as<int>());
        int h = 0;
        DT_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h) fail(DT_ERR_TIMEOUT, "dt_gram_tc: a tensor-core wait timed out");
        s.finish();
    });
}

}  // extern "C"
