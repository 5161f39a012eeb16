// Learned warm start for dense HOOI (no counterpart in the reference, whose
// HOOI_ALS starts from random factors, template/algorithm/tucker/hooi_als.tpp:74-81).
//
// The network is a linear autoencoder over factor columns of length n: an
// encoder E (k x n) and a decoder D (n x k), trained on the columns of HOOI
// solutions of a tensor family so that D E u ~ u.  At its optimum span(D) is
// the k-dimensional subspace that best holds those factor columns.
//
// Training (all on the device, these kernels plus the library's FP64 GEMM):
//   H = E U,  R = D H - U,  loss = |R|^2 / N          (U: n x N columns)
//   dD = (2/N) R H^T,  dE = (2/N) (D^T R) U^T,  Adam on E and D.
// One training step is captured once as a CUDA graph and replayed; the Adam
// step counter lives in device memory so the replays need no host work.
//
// Inference (the warm start of one tensor X, every mode of size n):
//   Q = orth(D); sketch C = X x_1 Q^T x_2 Q^T ... (k^N values, one pass over X);
//   V_m = leading R_m eigenvectors of C_(m) C_(m)^T, refined by HOOI sweeps on
//   the small sketch C (the best Tucker factors inside span(Q)); U_m = Q V_m.
// The fits |C|^2/|X|^2 (the sketch) and |X x_m U_m^T|^2/|X|^2 (the initial
// factors) come back with the factors so the caller can fall back to HOSVD.
#include <cmath>
#include <cstring>
#include <vector>

#include "dt_kernels.cuh"

namespace dt {
namespace {

// R = DH - U and per-block partial sums of R^2.
__global__ void ws_residual_kernel(const double *DH, const double *__restrict__ U, int64_t total,
                                   double *R, double *__restrict__ part) {
    __shared__ double red[32];
    double s = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const double r = DH[e] - U[e];
        R[e] = r;
        s = fma(r, r, s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) part[blockIdx.x] = s;
    }
}

// loss = sum(part) / N, summed in a fixed order; also logged at loss_hist[step].
__global__ void ws_loss_kernel(const double *__restrict__ part, int nparts, double invN,
                               double *__restrict__ loss, double *__restrict__ loss_hist,
                               const int *__restrict__ step) {
    double s = 0.0;
    for (int i = 0; i < nparts; i++) s += part[i];
    loss[0] = s * invN;
    if (loss_hist) loss_hist[*step] = s * invN;
}

__global__ void ws_scale_kernel(double *__restrict__ x, int64_t n, double a) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        x[e] *= a;
}

// Adam (Kingma & Ba) on one parameter block; step[0] counts completed steps.
__global__ void ws_adam_kernel(double *__restrict__ p, const double *__restrict__ g,
                               double *__restrict__ m, double *__restrict__ v, int64_t n,
                               double lr, double b1, double b2, double eps,
                               const int *__restrict__ step) {
    const int t = *step + 1;
    const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const double gi = g[e];
        const double mi = b1 * m[e] + (1.0 - b1) * gi;
        const double vi = b2 * v[e] + (1.0 - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        p[e] -= lr * (mi / c1) / (sqrt(vi / c2) + eps);
    }
}

__global__ void ws_step_kernel(int *step) { step[0] += 1; }

// splitmix64 -> uniform (0, 1] -> Box-Muller; host-side initial weights and
// eigen-solver starts.
struct HostGauss {
    uint64_t s;
    explicit HostGauss(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct WsBuffers {
    DevMem H, R, T, part, loss, gE, gD;
    int nparts = 0;
};

void ws_forward_backward(dt_ctx *ctx, const double *U, int64_t n, int64_t N, int k,
                         const double *E, const double *D, WsBuffers &b, double *loss_hist,
                         const int *step) {
    // H = E U (k x N)
    gemm_f64(ctx, 0, 0, k, N, n, E, k, U, n, b.H.as<double>(), k, 0.0);
    // R = D H (n x N), then R - U with the loss
    gemm_f64(ctx, 0, 0, n, N, k, D, n, b.H.as<double>(), k, b.R.as<double>(), n, 0.0);
    const int64_t total = n * N;
    DT_LAUNCH(ctx, ws_residual_kernel, b.nparts, 256, 0, b.R.as<double>(), U, total,
              b.R.as<double>(), b.part.as<double>());
    DT_LAUNCH(ctx, ws_loss_kernel, 1, 1, 0, b.part.as<double>(), b.nparts, 1.0 / (double)N,
              b.loss.as<double>(), loss_hist, step);
    const unsigned sb = std::max(1u, std::min<unsigned>(ceil_div(total, 256), 8u * ctx->num_sms));
    DT_LAUNCH(ctx, ws_scale_kernel, sb, 256, 0, b.R.as<double>(), total, 2.0 / (double)N);
    // dD = R' H^T (n x k); T = D^T R' (k x N); dE = T U^T (k x n)
    gemm_f64(ctx, 0, 1, n, k, N, b.R.as<double>(), n, b.H.as<double>(), k, b.gD.as<double>(), n,
             0.0);
    gemm_f64(ctx, 1, 0, k, N, n, D, n, b.R.as<double>(), n, b.T.as<double>(), k, 0.0);
    gemm_f64(ctx, 0, 1, k, n, N, b.T.as<double>(), k, U, n, b.gE.as<double>(), k, 0.0);
}

void ws_alloc(dt_ctx *ctx, int64_t n, int64_t N, int k, WsBuffers &b) {
    b.nparts = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n * N, 256), 4 * ctx->num_sms));
    b.H.alloc(ctx, (size_t)k * N * sizeof(double));
    b.R.alloc(ctx, (size_t)n * N * sizeof(double));
    b.T.alloc(ctx, (size_t)k * N * sizeof(double));
    b.part.alloc(ctx, (size_t)b.nparts * sizeof(double));
    b.loss.alloc(ctx, sizeof(double));
    b.gE.alloc(ctx, (size_t)k * n * sizeof(double));
    b.gD.alloc(ctx, (size_t)n * k * sizeof(double));
}

void check_model(int64_t n, int64_t N, int k) {
    DT_CHECK_ARG(n >= 1 && N >= 1, "warm start: need n >= 1 and N >= 1");
    DT_CHECK_ARG(k >= 1 && k <= 32 && k <= n, "warm start: need 1 <= k <= min(32, n) (k=%d)", k);
}

}  // namespace
}  // namespace dt

using namespace dt;

extern "C" {

int dt_ws_loss_grad(dt_ctx *ctx, const double *U, int64_t n, int64_t N, int k, const double *E,
                    const double *D, double *loss, double *gE, double *gD) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(U && E && D && loss && gE && gD, "dt_ws_loss_grad: null argument");
        check_model(n, N, k);
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView u(ctx, U, (size_t)n * N * sizeof(double), true, false);
        DevView e(ctx, E, (size_t)k * n * sizeof(double), true, false);
        DevView d(ctx, D, (size_t)n * k * sizeof(double), true, false);
        DevView l(ctx, loss, sizeof(double), false, true);
        DevView ge(ctx, gE, (size_t)k * n * sizeof(double), false, true);
        DevView gd(ctx, gD, (size_t)n * k * sizeof(double), false, true);
        WsBuffers b;
        ws_alloc(ctx, n, N, k, b);
        DevMem step(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(step.get(), 0, sizeof(int), ctx->stream));
        ws_forward_backward(ctx, u.as<double>(), n, N, k, e.as<double>(), d.as<double>(), b,
                            nullptr, step.as<int>());
        DT_CUDA(cudaMemcpyAsync(l.ptr(), b.loss.get(), sizeof(double), cudaMemcpyDeviceToDevice,
                                ctx->stream));
        DT_CUDA(cudaMemcpyAsync(ge.ptr(), b.gE.get(), (size_t)k * n * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        DT_CUDA(cudaMemcpyAsync(gd.ptr(), b.gD.get(), (size_t)n * k * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        l.finish();
        ge.finish();
        gd.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_ws_train(dt_ctx *ctx, const double *U, int64_t n, int64_t N, int k, int steps, double lr,
                uint64_t seed, double *E, double *D, double *loss_hist) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(U && E && D, "dt_ws_train: null argument");
        check_model(n, N, k);
        DT_CHECK_ARG(steps >= 0 && steps <= (1 << 24), "dt_ws_train: bad step count %d", steps);
        DT_CHECK_ARG(lr > 0.0, "dt_ws_train: learning rate must be positive");
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView u(ctx, U, (size_t)n * N * sizeof(double), true, false);
        DevView e(ctx, E, (size_t)k * n * sizeof(double), false, true);
        DevView d(ctx, D, (size_t)n * k * sizeof(double), false, true);
        // Gaussian initial weights, scale 1/sqrt(n) (E) and 1/sqrt(k) (D).
        {
            HostGauss g(seed);
            std::vector<double> he((size_t)k * n), hd((size_t)n * k);
            for (auto &x : he) x = g.normal() / std::sqrt((double)n);
            for (auto &x : hd) x = g.normal() / std::sqrt((double)k);
            DT_CUDA(cudaMemcpyAsync(e.ptr(), he.data(), he.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
            DT_CUDA(cudaMemcpyAsync(d.ptr(), hd.data(), hd.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
            DT_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        WsBuffers b;
        ws_alloc(ctx, n, N, k, b);
        const int64_t pe = (int64_t)k * n;
        DevMem mE(ctx, pe * sizeof(double)), vE(ctx, pe * sizeof(double));
        DevMem mD(ctx, pe * sizeof(double)), vD(ctx, pe * sizeof(double));
        DevMem step(ctx, sizeof(int)), hist(ctx, std::max(steps, 1) * sizeof(double));
        DT_CUDA(cudaMemsetAsync(mE.get(), 0, pe * sizeof(double), ctx->stream));
        DT_CUDA(cudaMemsetAsync(vE.get(), 0, pe * sizeof(double), ctx->stream));
        DT_CUDA(cudaMemsetAsync(mD.get(), 0, pe * sizeof(double), ctx->stream));
        DT_CUDA(cudaMemsetAsync(vD.get(), 0, pe * sizeof(double), ctx->stream));
        DT_CUDA(cudaMemsetAsync(step.get(), 0, sizeof(int), ctx->stream));
        const double b1 = 0.9, b2 = 0.999, eps = 1e-12;
        const unsigned ab = std::max(1u, std::min<unsigned>(ceil_div(pe, 256), 256u));
        auto one_step = [&] {
            ws_forward_backward(ctx, u.as<double>(), n, N, k, e.as<double>(), d.as<double>(), b,
                                hist.as<double>(), step.as<int>());
            DT_LAUNCH(ctx, ws_adam_kernel, ab, 256, 0, e.as<double>(), b.gE.as<double>(),
                      mE.as<double>(), vE.as<double>(), pe, lr, b1, b2, eps, step.as<int>());
            DT_LAUNCH(ctx, ws_adam_kernel, ab, 256, 0, d.as<double>(), b.gD.as<double>(),
                      mD.as<double>(), vD.as<double>(), pe, lr, b1, b2, eps, step.as<int>());
            DT_LAUNCH(ctx, ws_step_kernel, 1, 1, 0, step.as<int>());
        };
        const bool capturable = ctx->stream != nullptr && ctx->stream != cudaStreamLegacy &&
                                ctx->stream != cudaStreamPerThread;
        if (steps > 0 && !capturable) {
            for (int s = 0; s < steps; s++) one_step();
        } else if (steps > 0) {
            // Capture one step (split-K scratch of the GEMMs is allocated
            // inside the graph), then replay it.
            const int64_t l0 = ctx->launches;
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            DT_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            try {
                one_step();
            } catch (...) {
                cudaStreamEndCapture(ctx->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            DT_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
            const int64_t per_step = ctx->launches - l0;
            ctx->launches = l0;
            cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            DT_CUDA(err);
            for (int s = 0; s < steps; s++) {
                err = cudaGraphLaunch(exec, ctx->stream);
                if (err != cudaSuccess) break;
                ctx->launches += per_step;
            }
            cudaGraphExecDestroy(exec);
            DT_CUDA(err);
        }
        if (loss_hist && steps > 0) {
            DT_CUDA(cudaMemcpyAsync(loss_hist, hist.get(), steps * sizeof(double),
                                    cudaMemcpyDefault, ctx->stream));
        }
        e.finish();
        d.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_ws_init(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
               const int64_t *ranks, const double *D, int k, int sketch_sweeps, double *const *U,
               double *fit_sketch, double *fit_init) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(X && shape && ranks && D && U, "dt_ws_init: null argument");
        DT_CHECK_ARG(dtype == DT_F64 || dtype == DT_F32, "dt_ws_init: bad dtype %d", dtype);
        DT_CHECK_ARG(ndim >= 2 && ndim <= 8, "dt_ws_init: ndim %d not in [2, 8]", ndim);
        const int64_t n = shape[0];
        check_model(n, 1, k);
        for (int m = 0; m < ndim; m++) {
            DT_CHECK_ARG(shape[m] == n, "dt_ws_init: every mode must have the model's size %lld",
                         (long long)n);
            DT_CHECK_ARG(ranks[m] >= 1 && ranks[m] <= k,
                         "dt_ws_init: need 1 <= R_%d <= k (R=%lld, k=%d)", m,
                         (long long)ranks[m], k);
            DT_CHECK_ARG(U[m], "dt_ws_init: null factor %d", m);
        }
        DT_CUDA(cudaSetDevice(ctx->device));
        const int64_t xsize = prod(shape, ndim);
        const size_t esz = dtype == DT_F64 ? 8 : 4;
        DevView x(ctx, X, xsize * esz, true, false);
        DevView dv(ctx, D, (size_t)n * k * sizeof(double), true, false);
        DevMem Q(ctx, (size_t)n * k * sizeof(double));
        {
            const double *a[1] = {dv.as<double>()};
            double *q[1] = {Q.as<double>()};
            const int64_t mm[1] = {n}, kk[1] = {k};
            orth_batch(ctx, 1, a, q, mm, kk);
        }
        DevMem scal(ctx, 3 * sizeof(double));
        sumsq(ctx, x.ptr(), dtype, xsize, scal.as<double>());
        // Sketch C = X x_m Q^T for every mode (highest mode first).
        int64_t cur[8];
        std::memcpy(cur, shape, ndim * sizeof(int64_t));
        DevMem a, bbuf;
        const void *src = x.ptr();
        bool f32 = dtype == DT_F32;
        for (int m = ndim - 1; m >= 0; m--) {
            int64_t L = 1, B = 1;
            for (int p = 0; p < m; p++) L *= cur[p];
            for (int p = m + 1; p < ndim; p++) B *= cur[p];
            DevMem out(ctx, (size_t)L * k * B * sizeof(double));
            if (f32)
                ttm_f64<float>(ctx, static_cast<const float *>(src), L, cur[m], B, Q.as<double>(),
                               n, 1, k, out.as<double>());
            else
                ttm_f64<double>(ctx, static_cast<const double *>(src), L, cur[m], B,
                                Q.as<double>(), n, 1, k, out.as<double>());
            cur[m] = k;
            a = std::move(out);
            src = a.get();
            f32 = false;
        }
        const int64_t csize = prod(cur, ndim);
        sumsq(ctx, a.get(), DT_F64, csize, scal.as<double>() + 1);
        // Leading eigenvectors of each sketch unfolding's Gram, decoded by Q.
        DT_CHECK_ARG(sketch_sweeps >= 0, "dt_ws_init: sketch_sweeps must be >= 0");
        DevMem S(ctx, (size_t)k * k * sizeof(double));
        DevMem work(ctx, (3 * (size_t)k * k + k + 64) * sizeof(double)), flag(ctx, sizeof(int));
        DT_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), ctx->stream));
        std::vector<DevMem> Vm(ndim);
        for (int m = 0; m < ndim; m++) {
            int64_t L = 1, B = 1;
            for (int p = 0; p < m; p++) L *= k;
            for (int p = m + 1; p < ndim; p++) B *= k;
            ttt_f64(ctx, a.as<double>(), a.as<double>(), L, k, k, B, S.as<double>());
            HostGauss g(0x5EED0000ull + (uint64_t)m);
            std::vector<double> hv((size_t)k * ranks[m]);
            for (auto &v : hv) v = g.normal();
            Vm[m].alloc(ctx, hv.size() * sizeof(double));
            DT_CUDA(cudaMemcpyAsync(Vm[m].get(), hv.data(), hv.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
            subspace_iter(ctx, S.as<double>(), k, Vm[m].as<double>(), ranks[m], 60,
                          work.as<double>(), flag.as<int>());
            DT_CUDA(cudaStreamSynchronize(ctx->stream));  // the host start is reused
        }
        // HOOI on the sketch: the best rank-R Tucker factors inside span(Q).
        if (sketch_sweeps > 0) {
            dt_hooi_opts o;
            dt_hooi_default_opts(&o);
            o.init = DT_INIT_GIVEN;
            o.max_sweeps = sketch_sweeps;
            o.tol = 1e-14;
            double *vp[8];
            for (int m = 0; m < ndim; m++) vp[m] = Vm[m].as<double>();
            if (dt_hooi_dense(ctx, a.get(), DT_F64, ndim, cur, ranks, &o, nullptr, vp, nullptr) !=
                DT_OK)
                fail(DT_ERR_CUDA, std::string("dt_ws_init: sketch HOOI failed: ") + dt_last_error());
        }
        std::vector<DevView> uv;
        uv.reserve(ndim);
        for (int m = 0; m < ndim; m++) {
            uv.emplace_back(ctx, U[m], (size_t)n * ranks[m] * sizeof(double), false, true);
            gemm_f64(ctx, 0, 0, n, ranks[m], k, Q.as<double>(), n, Vm[m].as<double>(), k,
                     uv.back().as<double>(), n, 0.0);
        }
        // Fit of the initial factors: |X x_m U_m^T|^2.
        std::memcpy(cur, shape, ndim * sizeof(int64_t));
        src = x.ptr();
        f32 = dtype == DT_F32;
        for (int m = ndim - 1; m >= 0; m--) {
            int64_t L = 1, B = 1;
            for (int p = 0; p < m; p++) L *= cur[p];
            for (int p = m + 1; p < ndim; p++) B *= cur[p];
            DevMem out(ctx, (size_t)L * ranks[m] * B * sizeof(double));
            if (f32)
                ttm_f64<float>(ctx, static_cast<const float *>(src), L, cur[m], B,
                               uv[m].as<double>(), n, 1, ranks[m], out.as<double>());
            else
                ttm_f64<double>(ctx, static_cast<const double *>(src), L, cur[m], B,
                                uv[m].as<double>(), n, 1, ranks[m], out.as<double>());
            cur[m] = ranks[m];
            bbuf = std::move(out);
            src = bbuf.get();
            f32 = false;
        }
        sumsq(ctx, bbuf.get(), DT_F64, prod(ranks, ndim), scal.as<double>() + 2);
        double h[3];
        DT_CUDA(cudaMemcpyAsync(h, scal.get(), sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        for (auto &v : uv) v.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        DT_CHECK_ARG(h[0] > 0.0, "dt_ws_init: X is zero");
        if (fit_sketch) *fit_sketch = h[1] / h[0];
        if (fit_init) *fit_init = h[2] / h[0];
    });
}

}  // extern "C"
