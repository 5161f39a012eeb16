// Batched dense HOOI: many small 3-way tensors of uneven shapes and ranks
// decomposed in one persistent launch.
//
// Each CTA pulls tensors from an atomic work queue and runs the whole HOOI
// for one tensor at a time: the dimension-tree TTM chain (X x_3 U_3^T shared by
// modes 1 and 2, X x_1 U_1^T x_2 U_2^T for mode 3), the Gram Y_(n) Y_(n)^T,
// the five-step subspace iteration of ALS_ (hooi_als.tpp:7-34) with
// CholeskyQR, and finally the FP64 core and relative error.  X is read from
// global memory (it stays in L2 while its CTA works on it), Y_(n), the Gram
// and the factors live in shared memory, and the one large intermediate
// (I_1 x I_2 x R_3) in a per-CTA slice of global scratch.  Arithmetic is FP64
// throughout; X may be FP32.
//
// The block size is chosen by an autotuner (timing each candidate on a sample
// of the batch, cached per batch signature), and the launch (queue reset +
// persistent kernel) is captured into a CUDA graph and replayed as one unit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "dt_kernels.cuh"

namespace dt {
namespace {

constexpr int BMAX_I = 64;   // largest mode size
constexpr int BMAX_R = 8;    // largest rank

struct BatchArgs {
    int count;
    const int64_t *shape;     // count x 3
    const int64_t *rank;      // count x 3
    const float *X;
    const int64_t *xoff;      // element offsets of each tensor
    double *U;                // factors, I_n x R_n col-major blocks
    const int64_t *uoff;      // count x 3 element offsets
    double *G;                // cores
    const int64_t *goff;
    double *relerr;
    int sweeps, inner;
    double *scratch;          // gridDim.x x (BMAX_I^2 * BMAX_R) doubles
    int *queue;
};

__device__ double bsum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (l == 0) red[32] = v;
    }
    __syncthreads();
    return red[32];
}

// Cholesky of the r x r Gram in G (row-major, r <= 8) by lane c owning column
// c; overwrites G with R (upper).  Returns false on a non-positive pivot.
__device__ bool warp_chol8(double *G, int r) {
    const int lane = threadIdx.x & 31;
    double g[BMAX_R];
#pragma unroll
    for (int i = 0; i < BMAX_R; i++) g[i] = (i < r && lane < r) ? G[i * r + lane] : 0.0;
    const double g00 = __shfl_sync(0xffffffffu, g[0], 0);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < BMAX_R; k++) {
        if (k >= r) break;
        const double d = __shfl_sync(0xffffffffu, g[k], k);
        if (!(d > 1e-28 * g00)) ok = false;
        const double rkk = sqrt(fmax(d, 1e-300));
        const double inv = 1.0 / rkk;
        if (lane > k) g[k] *= inv;
        if (lane == k) g[k] = rkk;
#pragma unroll
        for (int i = k + 1; i < BMAX_R; i++) {
            if (i >= r) break;
            const double rki = __shfl_sync(0xffffffffu, g[k], i);
            if (lane >= i) g[i] = fma(-rki, g[k], g[i]);
        }
    }
    if (lane < r) {
#pragma unroll
        for (int i = 0; i < BMAX_R; i++)
            if (i < r) G[i * r + lane] = i <= lane ? g[i] : 0.0;
    }
    __syncwarp();
    return ok;
}

// dst (n x r col-major) = orth(src) by CholeskyQR; Gs is r x r scratch.
// Falls back to modified Gram-Schmidt when the Gram is not positive definite.
__device__ void cholqr(const double *src, double *dst, int n, int r, double *Gs, int *bad) {
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int a = e / r, b = e % r;
        double s = 0.0;
        for (int k = 0; k < n; k++) s = fma(src[k + a * n], src[k + b * n], s);
        Gs[e] = s;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool ok = warp_chol8(Gs, r);
        if (threadIdx.x == 0) *bad = ok ? 0 : 1;
    }
    __syncthreads();
    if (!*bad) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double q[BMAX_R];
#pragma unroll
            for (int c = 0; c < BMAX_R; c++) {
                if (c >= r) break;
                double acc = src[i + c * n];
#pragma unroll
                for (int k = 0; k < BMAX_R; k++) {
                    if (k >= c) break;
                    acc = fma(-q[k], Gs[k * r + c], acc);
                }
                q[c] = acc / Gs[c * r + c];
                dst[i + c * n] = q[c];
            }
        }
        __syncthreads();
        return;
    }
    // Rank-deficient product: modified Gram-Schmidt with zero columns kept zero.
    if (threadIdx.x == 0) {
        for (int c = 0; c < r; c++) {
            for (int i = 0; i < n; i++) dst[i + c * n] = src[i + c * n];
            for (int p = 0; p < c; p++) {
                double d = 0.0;
                for (int i = 0; i < n; i++) d += dst[i + c * n] * dst[i + p * n];
                for (int i = 0; i < n; i++) dst[i + c * n] -= d * dst[i + p * n];
            }
            double nr = 0.0;
            for (int i = 0; i < n; i++) nr += dst[i + c * n] * dst[i + c * n];
            nr = sqrt(nr);
            for (int i = 0; i < n; i++) dst[i + c * n] = nr > 0 ? dst[i + c * n] / nr : 0.0;
        }
    }
    __syncthreads();
}

// Leading subspace of S (n x n) from L (n x r), `iters` steps, in place on L.
__device__ void subspace(const double *S, int n, double *L, int r, int iters, double *Z,
                         double *Gs, int *bad) {
    double *in = L, *out = Z;
    for (int it = 0; it < iters; it++) {
        for (int e = threadIdx.x; e < n * r; e += blockDim.x) {
            const int i = e % n, c = e / n;
            double acc = 0.0;
            for (int k = 0; k < n; k++) acc = fma(S[i + n * k], in[k + n * c], acc);
            out[e] = acc;
        }
        __syncthreads();
        cholqr(out, in, n, r, Gs, bad);
    }
    (void)out;
}

template <int NT>
__global__ void __launch_bounds__(NT) batched_hooi_kernel(BatchArgs a) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[33];
    __shared__ int bad;
    __shared__ int cur;
    double *Us = sm;                              // 3 x BMAX_I x BMAX_R
    double *Ys = Us + 3 * BMAX_I * BMAX_R;        // BMAX_I x BMAX_R^2
    double *Ss = Ys + BMAX_I * BMAX_R * BMAX_R;   // BMAX_I x BMAX_I
    double *Zs = Ss + BMAX_I * BMAX_I;            // BMAX_I x BMAX_R
    double *Gs = Zs + BMAX_I * BMAX_R;            // BMAX_R x BMAX_R
    double *T = a.scratch + (int64_t)blockIdx.x * BMAX_I * BMAX_I * BMAX_R;
    for (;;) {
        if (threadIdx.x == 0) cur = atomicAdd(a.queue, 1);
        __syncthreads();
        const int t = cur;
        __syncthreads();
        if (t >= a.count) break;
        const int I0 = (int)a.shape[3 * t], I1 = (int)a.shape[3 * t + 1], I2 = (int)a.shape[3 * t + 2];
        const int R0 = (int)a.rank[3 * t], R1 = (int)a.rank[3 * t + 1], R2 = (int)a.rank[3 * t + 2];
        const float *X = a.X + a.xoff[t];
        double *U0 = Us, *U1 = Us + BMAX_I * BMAX_R, *U2 = Us + 2 * BMAX_I * BMAX_R;
        double *ug[3] = {a.U + a.uoff[3 * t], a.U + a.uoff[3 * t + 1], a.U + a.uoff[3 * t + 2]};
        for (int e = threadIdx.x; e < I0 * R0; e += NT) U0[e] = ug[0][e];
        for (int e = threadIdx.x; e < I1 * R1; e += NT) U1[e] = ug[1][e];
        for (int e = threadIdx.x; e < I2 * R2; e += NT) U2[e] = ug[2][e];
        const int64_t nx = (int64_t)I0 * I1 * I2;
        double s = 0.0;
        for (int64_t e = threadIdx.x; e < nx; e += NT) s = fma((double)X[e], (double)X[e], s);
        const double x2 = bsum(s, red);
        const int I01 = I0 * I1;
        for (int sw = 0; sw < a.sweeps; sw++) {
            // T = X x_3 U_3^T  (I0 x I1 x R2)
            for (int p = threadIdx.x; p < I01; p += NT) {
                double acc[BMAX_R] = {};
                for (int i2 = 0; i2 < I2; i2++) {
                    const double x = X[p + (int64_t)I01 * i2];
#pragma unroll
                    for (int r = 0; r < BMAX_R; r++)
                        if (r < R2) acc[r] = fma(x, U2[i2 + I2 * r], acc[r]);
                }
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R2) T[p + I01 * r] = acc[r];
            }
            __syncthreads();
            // Mode 1: Y_(1)[i0, r1 + R1 r2] = sum_i1 T[i0, i1, r2] U1[i1, r1]
            for (int q = threadIdx.x; q < I0 * R2; q += NT) {
                const int i0 = q % I0, r2 = q / I0;
                double acc[BMAX_R] = {};
                for (int i1 = 0; i1 < I1; i1++) {
                    const double v = T[i0 + I0 * i1 + I01 * r2];
#pragma unroll
                    for (int r = 0; r < BMAX_R; r++)
                        if (r < R1) acc[r] = fma(v, U1[i1 + I1 * r], acc[r]);
                }
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R1) Ys[i0 + I0 * (r + R1 * r2)] = acc[r];
            }
            __syncthreads();
            {
                const int K = R1 * R2;
                for (int e = threadIdx.x; e < I0 * I0; e += NT) {
                    const int i = e % I0, j = e / I0;
                    double acc = 0.0;
                    for (int k = 0; k < K; k++) acc = fma(Ys[i + I0 * k], Ys[j + I0 * k], acc);
                    Ss[e] = acc;
                }
                __syncthreads();
                subspace(Ss, I0, U0, R0, a.inner, Zs, Gs, &bad);
            }
            // Mode 2: Y_(2)[i1, r0 + R0 r2] = sum_i0 T[i0, i1, r2] U0[i0, r0]
            for (int q = threadIdx.x; q < I1 * R2; q += NT) {
                const int i1 = q % I1, r2 = q / I1;
                double acc[BMAX_R] = {};
                for (int i0 = 0; i0 < I0; i0++) {
                    const double v = T[i0 + I0 * i1 + I01 * r2];
#pragma unroll
                    for (int r = 0; r < BMAX_R; r++)
                        if (r < R0) acc[r] = fma(v, U0[i0 + I0 * r], acc[r]);
                }
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R0) Ys[i1 + I1 * (r + R0 * r2)] = acc[r];
            }
            __syncthreads();
            {
                const int K = R0 * R2;
                for (int e = threadIdx.x; e < I1 * I1; e += NT) {
                    const int i = e % I1, j = e / I1;
                    double acc = 0.0;
                    for (int k = 0; k < K; k++) acc = fma(Ys[i + I1 * k], Ys[j + I1 * k], acc);
                    Ss[e] = acc;
                }
                __syncthreads();
                subspace(Ss, I1, U1, R1, a.inner, Zs, Gs, &bad);
            }
            // Mode 3 from X: T2 = X x_1 U0^T (R0 x I1 x I2), then Y_(3).
            const int R0I1 = R0 * I1;
            for (int q = threadIdx.x; q < I1 * I2; q += NT) {
                const int64_t base = (int64_t)I0 * q;
                double acc[BMAX_R] = {};
                for (int i0 = 0; i0 < I0; i0++) {
                    const double x = X[base + i0];
#pragma unroll
                    for (int r = 0; r < BMAX_R; r++)
                        if (r < R0) acc[r] = fma(x, U0[i0 + I0 * r], acc[r]);
                }
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R0) T[r + R0 * q] = acc[r];
            }
            __syncthreads();
            // Y_(3)[i2, r0 + R0 r1] = sum_i1 T2[r0, i1, i2] U1[i1, r1]
            for (int q = threadIdx.x; q < R0 * I2; q += NT) {
                const int r0 = q % R0, i2 = q / R0;
                double acc[BMAX_R] = {};
                for (int i1 = 0; i1 < I1; i1++) {
                    const double v = T[r0 + R0 * i1 + R0I1 * i2];
#pragma unroll
                    for (int r = 0; r < BMAX_R; r++)
                        if (r < R1) acc[r] = fma(v, U1[i1 + I1 * r], acc[r]);
                }
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R1) Ys[i2 + I2 * (r0 + R0 * r)] = acc[r];
            }
            __syncthreads();
            {
                const int K = R0 * R1;
                for (int e = threadIdx.x; e < I2 * I2; e += NT) {
                    const int i = e % I2, j = e / I2;
                    double acc = 0.0;
                    for (int k = 0; k < K; k++) acc = fma(Ys[i + I2 * k], Ys[j + I2 * k], acc);
                    Ss[e] = acc;
                }
                __syncthreads();
                subspace(Ss, I2, U2, R2, a.inner, Zs, Gs, &bad);
            }
        }
        // Core G[k + K r2] = sum_i2 Y_(3)[i2, k] U2[i2, r2] (the last Y_(3) and U2
        // are those of the final sweep), relative error in FP64.
        const int K = R0 * R1;
        double *Gout = a.G + a.goff[t];
        double g2 = 0.0;
        for (int e = threadIdx.x; e < K * R2; e += NT) {
            const int k = e % K, r2 = e / K;
            double acc = 0.0;
            for (int i2 = 0; i2 < I2; i2++) acc = fma(Ys[i2 + I2 * k], U2[i2 + I2 * r2], acc);
            Gout[e] = acc;
            g2 = fma(acc, acc, g2);
        }
        g2 = bsum(g2, red);
        if (threadIdx.x == 0) a.relerr[t] = sqrt(fmax(0.0, 1.0 - g2 / x2));
        for (int e = threadIdx.x; e < I0 * R0; e += NT) ug[0][e] = U0[e];
        for (int e = threadIdx.x; e < I1 * R1; e += NT) ug[1][e] = U1[e];
        for (int e = threadIdx.x; e < I2 * R2; e += NT) ug[2][e] = U2[e];
        __syncthreads();
    }
}

size_t batched_smem() {
    return (3 * BMAX_I * BMAX_R + BMAX_I * BMAX_R * BMAX_R + BMAX_I * BMAX_I + BMAX_I * BMAX_R +
            BMAX_R * BMAX_R) *
           sizeof(double);
}

void launch_batched(dt_ctx *ctx, int nt, const BatchArgs &a, unsigned grid) {
    const size_t smem = batched_smem();
    DT_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(int), ctx->stream));
    switch (nt) {
        case 128:
            smem_limit(ctx, batched_hooi_kernel<128>, smem);
            DT_LAUNCH(ctx, batched_hooi_kernel<128>, grid, 128, smem, a);
            break;
        case 512:
            smem_limit(ctx, batched_hooi_kernel<512>, smem);
            DT_LAUNCH(ctx, batched_hooi_kernel<512>, grid, 512, smem, a);
            break;
        default:
            smem_limit(ctx, batched_hooi_kernel<256>, smem);
            DT_LAUNCH(ctx, batched_hooi_kernel<256>, grid, 256, smem, a);
            break;
    }
}

unsigned batched_grid(dt_ctx *ctx, int nt) {
    // Resident CTAs per SM for this block size and the shared-memory footprint.
    int per_sm = 1;
    const size_t smem = batched_smem();
    if (nt == 128)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_hooi_kernel<128>, 128, smem);
    else if (nt == 512)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_hooi_kernel<512>, 512, smem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_hooi_kernel<256>, 256, smem);
    return (unsigned)(std::max(1, per_sm) * ctx->num_sms);
}

}  // namespace

// Per-context autotuning cache: block size chosen for each batch signature
// (count, largest mode, largest rank, sweeps, inner iterations).
struct BatchedState {
    std::map<std::vector<int64_t>, int> tuned;
};

static std::map<dt_ctx *, BatchedState> g_batched;

}  // namespace dt

using namespace dt;

extern "C" {

int dt_hooi_batched(dt_ctx *ctx, int count, const int64_t *shapes, const int64_t *ranks,
                    const float *X, const int64_t *x_offsets, int sweeps, int inner_iters,
                    double *U, const int64_t *u_offsets, double *G, const int64_t *g_offsets,
                    double *relerr, int block_threads, dt_batched_report *report) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(count >= 1 && shapes && ranks && X && x_offsets && U && u_offsets && G &&
                         g_offsets && relerr,
                     "dt_hooi_batched: bad arguments");
        DT_CHECK_ARG(sweeps >= 1 && inner_iters >= 1, "dt_hooi_batched: sweeps/inner must be >= 1");
        DT_CHECK_ARG(block_threads == 0 || block_threads == 128 || block_threads == 256 ||
                         block_threads == 512,
                     "dt_hooi_batched: block_threads must be 0 (autotune), 128, 256 or 512");
        int64_t xn = 0, un = 0, gn = 0;
        std::vector<int64_t> sig;
        int64_t maxI = 0, maxR = 0;
        for (int t = 0; t < count; t++) {
            int64_t xs = 1, gs = 1;
            for (int m = 0; m < 3; m++) {
                const int64_t I = shapes[3 * t + m], R = ranks[3 * t + m];
                DT_CHECK_ARG(I >= 1 && I <= BMAX_I && R >= 1 && R <= BMAX_R && R <= I,
                             "dt_hooi_batched: tensor %d mode %d: need 1 <= R <= I, I <= %d, R <= %d",
                             t, m, BMAX_I, BMAX_R);
                xs *= I;
                gs *= R;
                un = std::max(un, u_offsets[3 * t + m] + I * R);
                maxI = std::max(maxI, I);
                maxR = std::max(maxR, R);
            }
            xn = std::max(xn, x_offsets[t] + xs);
            gn = std::max(gn, g_offsets[t] + gs);
        }
        sig = {count, maxI, maxR, sweeps, inner_iters};
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView xv(ctx, X, xn * sizeof(float), true, false);
        DevView uv(ctx, U, un * sizeof(double), true, true);
        DevView gv(ctx, G, gn * sizeof(double), false, true);
        DevView ev(ctx, relerr, count * sizeof(double), false, true);
        auto cp = [&](const int64_t *h, size_t n, DevMem &d) {
            d.alloc(ctx, n * sizeof(int64_t));
            DT_CUDA(cudaMemcpyAsync(d.get(), h, n * sizeof(int64_t), cudaMemcpyHostToDevice,
                                    ctx->stream));
        };
        // Descriptor tables are cached with the graph: keep them in the state.
        BatchedState &st = g_batched[ctx];
        DevMem dshape, drank, dxoff, duoff, dgoff;
        cp(shapes, 3 * (size_t)count, dshape);
        cp(ranks, 3 * (size_t)count, drank);
        cp(x_offsets, count, dxoff);
        cp(u_offsets, 3 * (size_t)count, duoff);
        cp(g_offsets, count, dgoff);
        DevMem queue(ctx, sizeof(int));
        BatchArgs a{};
        a.count = count;
        a.shape = dshape.as<int64_t>();
        a.rank = drank.as<int64_t>();
        a.X = xv.as<float>();
        a.xoff = dxoff.as<int64_t>();
        a.U = uv.as<double>();
        a.uoff = duoff.as<int64_t>();
        a.G = gv.as<double>();
        a.goff = dgoff.as<int64_t>();
        a.relerr = ev.as<double>();
        a.sweeps = sweeps;
        a.inner = inner_iters;
        a.queue = queue.as<int>();
        int nt = block_threads;
        const int64_t launches0 = ctx->launches;
        double tune_ms[3] = {0, 0, 0};
        if (nt == 0) {
            auto it = st.tuned.find(sig);
            if (it != st.tuned.end()) {
                nt = it->second;
            } else {
                // Autotune on a sample of the batch with a scratch copy of U.
                const int sample = std::min(count, 512);
                DevMem ucopy(ctx, un * sizeof(double));
                const int cand[3] = {128, 256, 512};
                float best = 1e30f;
                for (int c = 0; c < 3; c++) {
                    BatchArgs b = a;
                    b.count = sample;
                    b.U = ucopy.as<double>();
                    const unsigned grid = batched_grid(ctx, cand[c]);
                    DevMem scratch(ctx, (size_t)grid * BMAX_I * BMAX_I * BMAX_R * sizeof(double));
                    b.scratch = scratch.as<double>();
                    DT_CUDA(cudaMemcpyAsync(ucopy.get(), uv.ptr(), un * sizeof(double),
                                            cudaMemcpyDeviceToDevice, ctx->stream));
                    launch_batched(ctx, cand[c], b, grid);  // warm
                    DT_CUDA(cudaMemcpyAsync(ucopy.get(), uv.ptr(), un * sizeof(double),
                                            cudaMemcpyDeviceToDevice, ctx->stream));
                    DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
                    launch_batched(ctx, cand[c], b, grid);
                    DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
                    DT_CUDA(cudaEventSynchronize(ctx->ev_stop));
                    float ms = 0.f;
                    DT_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
                    tune_ms[c] = ms;
                    if (ms < best) {
                        best = ms;
                        nt = cand[c];
                    }
                }
                st.tuned[sig] = nt;
            }
        }
        const unsigned grid = batched_grid(ctx, nt);
        DevMem scratch(ctx, (size_t)grid * BMAX_I * BMAX_I * BMAX_R * sizeof(double));
        a.scratch = scratch.as<double>();
        // Capture queue reset + persistent kernel into a graph, then replay it.
        cudaGraph_t graph;
        cudaGraphExec_t exec;
        DT_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const size_t smem = batched_smem();
        switch (nt) {
            case 128:
                smem_limit(ctx, batched_hooi_kernel<128>, smem);
                break;
            case 512:
                smem_limit(ctx, batched_hooi_kernel<512>, smem);
                break;
            default:
                smem_limit(ctx, batched_hooi_kernel<256>, smem);
        }
        cudaMemsetAsync(a.queue, 0, sizeof(int), ctx->stream);
        if (nt == 128)
            batched_hooi_kernel<128><<<grid, 128, smem, ctx->stream>>>(a);
        else if (nt == 512)
            batched_hooi_kernel<512><<<grid, 512, smem, ctx->stream>>>(a);
        else
            batched_hooi_kernel<256><<<grid, 256, smem, ctx->stream>>>(a);
        ctx->launches++;
        DT_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
        DT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        DT_CUDA(cudaGraphDestroy(graph));
        DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
        const cudaError_t le = cudaGraphLaunch(exec, ctx->stream);
        DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaGraphExecDestroy(exec);
        DT_CUDA(le);
        float ms = 0.f;
        DT_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        uv.finish();
        gv.finish();
        ev.finish();
        if (report) {
            std::memset(report, 0, sizeof(*report));
            report->device_ms = ms;
            report->block_threads = nt;
            report->grid = (int)grid;
            report->kernel_launches = (int)(ctx->launches - launches0);
            for (int c = 0; c < 3; c++) report->tune_ms[c] = tune_ms[c];
        }
    });
}

}  // extern "C"
