// Mixed-precision dense HOOI: the TTM chain and the Gram run on the tcgen05
// tensor cores in BF16 (optionally with hi+lo split operands) with FP32
// accumulation; the subspace iteration / QR, the fit subtraction and the
// final core projection stay in FP64.
//
// Schedule: sweeps in plain BF16 until the residual settles to the BF16 noise
// floor, then `refine_sweeps` sweeps with split hi+lo operands (~2^-16
// relative), then the core G = X x_1 U_1^T ... x_N U_N^T projected in FP64 from
// the original X.  DT_PREC_BF16X2 runs every sweep split.  The same dimension
// tree as the FP64 driver is used; each chain contracts its highest mode
// first so the non-contracted prefix (the TMA row dimension) stays long, and a
// leaf's last contraction writes Y_(n) K-major for the Gram.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "dt_hooi.cuh"
#include "dt_kernels.cuh"
#include "dt_tc_host.cuh"

namespace dt {
namespace {

__global__ void f64_to_f32_kernel(const double *__restrict__ x, int64_t n, float *__restrict__ y) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        y[e] = (float)x[e];
}

// The device-side sweep loop's state: sweeps done, the last residual, and
// the residual of every sweep.
struct LoopState {
    int it, pad;
    double prev;
    double hist[DT_MAX_HIST];
};

// End of one sweep of the device-side loop: the sweep's residual from its
// ||G||^2 and ||X||^2, the stop rule of the host loop (residual change below
// `thr`, or `max_sweeps` done), and the loop's condition for the next pass.
__global__ void sweep_check_kernel(cudaGraphConditionalHandle h, const double *scal,
                                   LoopState *st, double thr, int max_sweeps) {
    pdl_wait();
    const double x2 = scal[0], g2 = scal[1];
    const double res = sqrt(fmax(0.0, 1.0 - g2 / x2));
    const int it = st->it;
    if (it < DT_MAX_HIST) st->hist[it] = res;
    const bool stop = it + 1 >= max_sweeps || (thr > 0.0 && it > 0 && fabs(res - st->prev) < thr);
    st->prev = res;
    st->it = it + 1;
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// The whole sweep loop as one graph: a reset of the LoopState, then a WHILE
// node whose body is one captured sweep followed by sweep_check_kernel.
struct LoopGraph {
    cudaGraphExec_t exec = nullptr;
    bool failed = false;
    int64_t launches_per_sweep = 0;
    double thr = -1.0;
    int max_sweeps = -1;
    ~LoopGraph() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

// A BF16 intermediate of the sweep (hi, and lo when split), in the plan's
// arena.
struct BfTensor {
    __nv_bfloat16 *hi = nullptr, *lo = nullptr;
    int64_t shape[16];
};

struct MixedHooi {
    dt_ctx *ctx = nullptr;
    int N = 0;
    int64_t I[16] = {}, R[16] = {};
    int64_t xsize = 0;
    dt_hooi_opts opts{};
    const float *X32 = nullptr;
    DevMem X32own, Xh, Xl;
    std::vector<DevMem> U;
    DevMem S, work, flag, err, scal, Gs;
    bool split = false;   // intermediates, U and the Gram operands as hi + lo
    bool xsplit = false;  // X itself as hi + lo (else X in BF16 hi only)
    DenseHooi helper;  // initial factors (same generators as the FP64 driver)
    LaunchTimer *xtimer = nullptr;
    SweepGraph *g_bf16 = nullptr, *g_split = nullptr;  // captured sweeps (or null)
    // Sweep intermediates (tensors, Gram partial tiles, core partial sums) come
    // from one per-plan buffer used as a stack and handed out in the same order
    // every sweep, so a captured sweep sees the same addresses and holds no
    // allocation nodes.  A dry pass of the sweep (no launches) sizes it.
    DevMem arena;
    size_t arena_cap = 0, arena_off = 0, arena_need = 0;
    bool dry = false;
    LoopGraph *loop = nullptr;  // the device-side sweep loop (or null)
    DevMem loopst;              // its LoopState

    // Builds the device-side loop for split sweeps with stop threshold `thr`
    // and `max_sweeps`; false (and no further attempts) when the runtime
    // refuses any step, in which case the host drives the sweeps.
    bool build_loop(double thr, int max_sweeps) {
        LoopGraph &lg = *loop;
        if (lg.exec && lg.thr == thr && lg.max_sweeps == max_sweeps) return true;
        if (lg.failed) return false;
        if (lg.exec) {
            cudaGraphExecDestroy(lg.exec);
            lg.exec = nullptr;
        }
        if (!loopst.get()) loopst.alloc(ctx, sizeof(LoopState));
        cudaGraph_t g = nullptr;
        bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
        cudaGraphConditionalHandle h = 0;
        ok = ok && cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) ==
                       cudaSuccess;
        cudaGraphNode_t reset = nullptr, cond = nullptr;
        if (ok) {
            cudaMemsetParams mp = {};
            mp.dst = loopst.get();
            mp.value = 0;
            mp.elementSize = 4;
            mp.width = sizeof(LoopState) / 4;
            mp.height = 1;
            mp.pitch = 0;
            ok = cudaGraphAddMemsetNode(&reset, g, nullptr, 0, &mp) == cudaSuccess;
        }
        cudaGraphNodeParams cp = {};
        if (ok) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&cond, g, &reset, 1, &cp) == cudaSuccess;
        }
        const int64_t l0 = ctx->launches;
        if (ok) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            ok = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeRelaxed) == cudaSuccess;
            if (ok) {
                try {
                    sweep();
                    DT_LAUNCH_PDL(ctx, sweep_check_kernel, 1, 1, 0, h,
                              (const double *)scal.as<double>(), loopst.as<LoopState>(), thr,
                              max_sweeps);
                } catch (...) {
                    ok = false;
                }
                cudaGraph_t out = nullptr;
                ok = cudaStreamEndCapture(ctx->stream, &out) == cudaSuccess && ok;
            }
        }
        lg.launches_per_sweep = ctx->launches - l0;
        ctx->launches = l0;
        ok = ok && cudaGraphInstantiate(&lg.exec, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (!ok) {
            if (lg.exec) cudaGraphExecDestroy(lg.exec);
            lg.exec = nullptr;
            lg.failed = true;
            return false;
        }
        lg.thr = thr;
        lg.max_sweeps = max_sweeps;
        return true;
    }

    void *take(size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        const size_t off = arena_off;
        arena_off += bytes;
        arena_need = std::max(arena_need, arena_off);
        if (dry) return nullptr;
        if (arena_off > arena_cap)
            fail(DT_ERR_CUDA, fmt("internal: sweep arena of %zu bytes exceeded", arena_cap));
        return static_cast<char *>(arena.get()) + off;
    }

    // Sizes the arena for split sweeps (the larger kind) and allocates it.
    void size_arena() {
        const bool s0 = split;
        split = true;
        dry = true;
        arena_off = arena_need = 0;
        sweep();
        dry = false;
        split = s0;
        arena.alloc(ctx, arena_need);
        arena_cap = arena_need;
    }

    static std::vector<int> order_high_first(std::vector<int> modes) {
        std::sort(modes.begin(), modes.end(), [](int a, int b) { return a > b; });
        return modes;
    }

    static bool plan_ok_for(int n, const int64_t *shape, const int64_t *ranks) {
        MixedHooi t;
        t.N = n;
        for (int m = 0; m < n; m++) {
            t.I[m] = shape[m];
            t.R[m] = ranks[m];
        }
        return t.plan_ok();
    }

    // Checks every contraction and Gram of the dimension tree against the
    // tensor-core kernels' layout rules.
    bool plan_ok() const {
        if (N < 2 || N > 8) return false;
        for (int n = 0; n < N; n++) {
            int64_t K = 1;
            for (int m = 0; m < N; m++)
                if (m != n) K *= R[m];
            if (!tc_gram_supported(I[n], K) || R[n] > 32) return false;
        }
        std::vector<int64_t> sh(I, I + N);
        return node_ok(0, N, sh);
    }
    bool node_ok(int lo, int hi, std::vector<int64_t> sh) const {
        if (hi - lo == 1) return true;
        const int mid = (lo + hi + 1) / 2;  // [0,3) -> [0,2) + [2,3): long TMA rows
        for (int side = 0; side < 2; side++) {
            const int clo = side == 0 ? lo : mid, chi = side == 0 ? mid : hi;
            std::vector<int> modes;
            for (int m = lo; m < hi; m++)
                if (m < clo || m >= chi) modes.push_back(m);
            std::vector<int64_t> c = sh;
            for (int m : order_high_first(modes)) {
                int64_t L = 1, B = 1;
                for (int k = 0; k < m; k++) L *= c[k];
                for (int k = m + 1; k < N; k++) B *= c[k];
                if (!tc_ttm_supported(L, c[m], B, R[m])) return false;
                c[m] = R[m];
            }
            if (!node_ok(clo, chi, c)) return false;
        }
        return true;
    }

    // Contract `modes` of T; the last contraction of a leaf chain (leaf >= 0)
    // writes Y_(leaf) K-major.
    BfTensor contract_all(const __nv_bfloat16 *Th, const __nv_bfloat16 *Tl,
                          const int64_t *shape, std::vector<int> modes, int leaf) {
        BfTensor cur;
        std::memcpy(cur.shape, shape, N * sizeof(int64_t));
        const __nv_bfloat16 *sh = Th, *sl = Tl;
        const std::vector<int> ord = order_high_first(modes);
        for (size_t q = 0; q < ord.size(); q++) {
            const int m = ord[q];
            int64_t L = 1, B = 1;
            for (int k = 0; k < m; k++) L *= cur.shape[k];
            for (int k = m + 1; k < N; k++) B *= cur.shape[k];
            const int64_t outn = L * R[m] * B;
            BfTensor nxt;
            std::memcpy(nxt.shape, cur.shape, N * sizeof(int64_t));
            nxt.shape[m] = R[m];
            nxt.hi = static_cast<__nv_bfloat16 *>(take(outn * sizeof(__nv_bfloat16)));
            if (split) nxt.lo = static_cast<__nv_bfloat16 *>(take(outn * sizeof(__nv_bfloat16)));
            OutMap om;
            const bool last_of_leaf = leaf >= 0 && q + 1 == ord.size();
            if (!last_of_leaf) {
                om.nl = 1;
                om.dl[0] = std::max<int64_t>(L, 1);
                om.sl[0] = 1;
                om.nb = 1;
                om.db[0] = std::max<int64_t>(B, 1);
                om.sb[0] = L * R[m];
                om.jstride = L;
            } else {
                // Y_(leaf)[t_leaf][k], k = sum_{q != leaf} t_q * kst_q.
                int64_t kst[16], K = 1;
                for (int p = 0; p < N; p++) {
                    if (p == leaf) continue;
                    kst[p] = K;
                    K *= nxt.shape[p];
                }
                kst[leaf] = K;
                om.nl = m;
                for (int p = 0; p < m; p++) {
                    om.dl[p] = cur.shape[p];
                    om.sl[p] = kst[p];
                }
                om.nb = N - m - 1;
                for (int p = m + 1; p < N; p++) {
                    om.db[p - m - 1] = cur.shape[p];
                    om.sb[p - m - 1] = kst[p];
                }
                om.jstride = kst[m];
                if (om.nl == 0) {
                    om.nl = 1;
                    om.dl[0] = 1;
                    om.sl[0] = 0;
                }
                if (om.nb == 0) {
                    om.nb = 1;
                    om.db[0] = 1;
                    om.sb[0] = 0;
                }
            }
            const bool is_x = sh == Xh.as<__nv_bfloat16>();
            const bool from_x = xtimer && is_x && !dry;
            // X is read as hi + lo only when xsplit; every other operand, U and
            // the output follow `split`.
            const __nv_bfloat16 *a_lo = split && (!is_x || xsplit) ? sl : nullptr;
            if (from_x) xtimer->begin();
            if (!dry)
                tc_ttm(ctx, sh, a_lo, L, cur.shape[m], B, U[m].as<double>(), R[m], om, nxt.hi,
                       split ? nxt.lo : nullptr, nullptr, err.as<int>(), split ? 1 : 0);
            if (from_x)
                xtimer->end((double)L * cur.shape[m] * B * 2 * (a_lo ? 2 : 1) +
                            (double)L * R[m] * B * 2 * (split ? 2 : 1) +
                            (double)cur.shape[m] * R[m] * 8);
            cur = nxt;
            sh = cur.hi;
            sl = split ? cur.lo : nullptr;
        }
        return cur;
    }

    void leaf(int n, const BfTensor &Y) {
        int64_t K = 1;
        for (int m = 0; m < N; m++)
            if (m != n) K *= R[m];
        const __nv_bfloat16 *yh = Y.hi;
        const __nv_bfloat16 *yl = split ? Y.lo : nullptr;
        void *gscr = take(tc_gram_scratch_bytes(I[n], K, split));
        void *cscr = n == N - 1 ? take(core_rows_scratch_bytes(K)) : nullptr;
        if (dry) return;
        tc_gram(ctx, yh, yl, I[n], K, S.as<double>(), err.as<int>(), gscr);
        subspace_iter(ctx, S.as<double>(), I[n], U[n].as<double>(), R[n], opts.inner_iters,
                      work.as<double>(), flag.as<int>());
        if (n == N - 1)
            core_rows(ctx, yh, yl, I[n], K, U[n].as<double>(), R[n], Gs.as<double>(),
                      scal.as<double>() + 1, cscr);
    }

    void node(int lo, int hi, const __nv_bfloat16 *Th, const __nv_bfloat16 *Tl,
              const int64_t *shape) {
        const int mid = (lo + hi + 1) / 2;  // [0,3) -> [0,2) + [2,3): long TMA rows
        for (int side = 0; side < 2; side++) {
            const int clo = side == 0 ? lo : mid, chi = side == 0 ? mid : hi;
            std::vector<int> modes;
            for (int m = lo; m < hi; m++)
                if (m < clo || m >= chi) modes.push_back(m);
            const bool is_leaf = chi - clo == 1;
            // The arena is a stack: what a side allocates is released once
            // the side is done, and the next side writes over it.
            const size_t mark = arena_off;
            BfTensor child = contract_all(Th, Tl, shape, modes, is_leaf ? clo : -1);
            if (is_leaf)
                leaf(clo, child);
            else
                node(clo, chi, child.hi, split ? child.lo : nullptr, child.shape);
            arena_off = mark;
        }
    }

    void sweep() {
        arena_off = 0;
        node(0, N, Xh.as<__nv_bfloat16>(), split && xsplit ? Xl.as<__nv_bfloat16>() : nullptr, I);
    }

    // 2 |X| R per X pass: each half of the tree first contracts its highest
    // mode.
    double x_pass_flop() const {
        const int mid = (N + 1) / 2;
        return 2.0 * xsize * (R[N - 1] + R[mid - 1]);
    }

    // Through the context's pinned block: an asynchronous copy and one
    // synchronisation.
    void read_scalars(int k, int n, double *out) {
        double *st = static_cast<double *>(host_stage(ctx));
        DT_CUDA(cudaMemcpyAsync(st, scal.as<double>() + k, n * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        std::memcpy(out, st, n * sizeof(double));
    }

    double read_scalar(int k) {
        double h = 0.0;
        read_scalars(k, 1, &h);
        return h;
    }

    void run(const void *X, int dtype, double *G_user, double *const *U_user,
             dt_hooi_report *rep, const ChunkedUpload *upload) {
        const int64_t launches0 = ctx->launches;
        LaunchTimer timer(ctx, opts.profile != 0);
        xtimer = &timer;
        // Whether X itself is kept as hi + lo: the split sweeps of DT_PREC_BF16X2
        // and of DT_PREC_BF16's refinement read both halves; DT_PREC_BF16XH
        // reads X in BF16 only (its intermediates, U and Grams are split).
        const bool want_split = opts.precision == DT_PREC_BF16X2 ||
                                (opts.precision == DT_PREC_BF16 && opts.refine_sweeps > 0);
        xsplit = want_split;
        DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
        if (dtype == DT_F32) {
            X32 = static_cast<const float *>(X);
        } else {
            X32own.alloc(ctx, xsize * sizeof(float));
            const unsigned blocks = std::max(1u, std::min<unsigned>(ceil_div(xsize, 256), 8u * ctx->num_sms));
            DT_LAUNCH(ctx, f64_to_f32_kernel, blocks, 256, 0, static_cast<const double *>(X), xsize,
                      X32own.as<float>());
            X32 = X32own.as<float>();
        }
        // Xh / Xl persist with the plan (the captured sweeps read them).
        if (!Xh.get()) Xh.alloc(ctx, xsize * sizeof(__nv_bfloat16));
        if (want_split && !Xl.get()) Xl.alloc(ctx, xsize * sizeof(__nv_bfloat16));
        if (dtype == DT_F64)
            sumsq(ctx, X, DT_F64, xsize, scal.as<double>());
        DevMem x2f(ctx, sizeof(double));
        if (upload)
            split_f32_chunks(ctx, *upload, Xh.as<__nv_bfloat16>(),
                             want_split ? Xl.as<__nv_bfloat16>() : nullptr, scal.as<double>());
        else
            split_f32(ctx, X32, xsize, Xh.as<__nv_bfloat16>(),
                      want_split ? Xl.as<__nv_bfloat16>() : nullptr,
                      dtype == DT_F32 ? scal.as<double>() : x2f.as<double>());
        // Initial factors: the FP64 driver's generators (libc Gaussian + QR,
        // or the caller's); HOSVD is not offered on this path.
        {
            double *dst[16];
            for (int m = 0; m < N; m++) dst[m] = U[m].as<double>();
            helper.init_factors(U_user, dst);
        }
        // ||X||^2 is read with the first sweep's ||G||^2 (one synchronisation).
        double x2 = -1.0;
        // Phases: BF16 sweeps until the residual settles to the BF16 noise
        // floor (kBf16Settle) or kBf16Max sweeps, then split hi+lo sweeps:
        // `refine_sweeps` of them (DT_PREC_BF16), or until the residual
        // settles to max(tol, kSplitFloor) (DT_PREC_BF16X2).  The residual a
        // sweep tracks comes from its own low-precision core, so the floors
        // sit above that noise; the reported residual is the FP64 projection.
        constexpr double kBf16Settle = 1e-3, kSplitFloor = 5e-6;
        constexpr int kBf16Max = 8;
        double prev = -1.0, res = 0.0;
        int sweeps = 0, bf16_done = 0, split_done = 0;
        const bool refine_mode = opts.precision == DT_PREC_BF16;
        split = opts.precision == DT_PREC_BF16X2 || opts.precision == DT_PREC_BF16XH;
        // Split sweeps throughout: the loop and its stop test run on the
        // device as one graph launch (no synchronisation per sweep), unless
        // per-sweep host work is asked for (profiling, verbose output, the
        // Summary profiler) or the stream cannot be captured.
        const bool plain_stream = ctx->stream != nullptr && ctx->stream != cudaStreamLegacy &&
                                  ctx->stream != cudaStreamPerThread;
        const bool device_loop = split && !refine_mode && loop && plain_stream &&
                                 graphs_enabled() && !opts.profile && !opts.verbose &&
                                 !summary_active(ctx) && opts.max_sweeps >= 1 &&
                                 build_loop(opts.tol > 0 ? std::max(opts.tol, kSplitFloor) : 0.0,
                                            opts.max_sweeps);
        if (device_loop) DT_CUDA(cudaGraphLaunch(loop->exec, ctx->stream));
        for (int it = 0; it < (device_loop ? 0 : opts.max_sweeps); it++) {
            if (!split && refine_mode && opts.refine_sweeps > 0 &&
                it >= opts.max_sweeps - opts.refine_sweeps) {
                split = true;
                prev = -1.0;
            }
            {
                // Counted work: the sweep's two passes over X (3 products per
                // element and rank with split operands).
                SummaryScope sc(ctx, split ? "HOOI sweep (BF16 split)" : "HOOI sweep (BF16)",
                                x_pass_flop() * (split ? (xsplit ? 3 : 2) : 1),
                                2.0 * xsize * (split && xsplit ? 4 : 2));
                SweepGraph *gr = split ? g_split : g_bf16;
                if (gr && !opts.profile)
                    gr->run(ctx, [&] { sweep(); });
                else
                    sweep();
            }
            double g2;
            if (x2 < 0.0) {
                double xg[2];
                read_scalars(0, 2, xg);
                x2 = xg[0];
                g2 = xg[1];
            } else {
                g2 = read_scalar(1);
            }
            res = std::sqrt(std::max(0.0, 1.0 - g2 / x2));
            if (rep && it < DT_MAX_HIST) rep->res_hist[it] = res;
            sweeps = it + 1;
            if (opts.verbose)
                fprintf(stderr, "[dt_hooi bf16%s] sweep %d  residual = %.12e\n",
                        split ? (xsplit ? "x2" : "xh") : "", it + 1, res);
            const double delta = prev >= 0 ? std::fabs(res - prev) : 1e300;
            prev = res;
            if (!split) {
                bf16_done++;
                const bool settled = delta < kBf16Settle || bf16_done >= kBf16Max;
                if (opts.refine_sweeps > 0 && settled) {
                    split = true;
                    prev = -1.0;
                } else if (opts.refine_sweeps == 0 && opts.tol > 0 && delta < std::max(opts.tol, kBf16Settle)) {
                    break;
                }
            } else {
                split_done++;
                if (refine_mode) {
                    if (split_done >= opts.refine_sweeps) break;
                    if (opts.tol > 0 && delta < std::max(opts.tol, kSplitFloor)) break;
                } else if (opts.tol > 0 && delta < std::max(opts.tol, kSplitFloor)) {
                    break;
                }
            }
        }
        if (x2 < 0.0 && !device_loop) x2 = read_scalar(0);
        // Final core, FP64 projection from the original X (the returned G is
        // X x_1 U_1^T ... x_N U_N^T to FP64 rounding).
        DevMem cur;
        {
            SummaryScope sc(ctx, "core projection (FP64)", 2.0 * xsize * R[N - 1],
                            4.0 * xsize);
            int64_t shape[16];
            std::memcpy(shape, I, N * sizeof(int64_t));
            std::vector<int> ord(N);
            std::iota(ord.begin(), ord.end(), 0);
            std::sort(ord.begin(), ord.end(), [](int a, int b) { return a > b; });
            const void *src = X32;
            bool src_f32 = true;
            for (int m : ord) {
                int64_t L = 1, B = 1;
                for (int k = 0; k < m; k++) L *= shape[k];
                for (int k = m + 1; k < N; k++) B *= shape[k];
                DevMem nxt(ctx, L * R[m] * B * sizeof(double));
                if (src_f32)
                    ttm_f64<float>(ctx, static_cast<const float *>(src), L, shape[m], B,
                                   U[m].as<double>(), I[m], 1, R[m], nxt.as<double>());
                else
                    ttm_f64<double>(ctx, static_cast<const double *>(src), L, shape[m], B,
                                    U[m].as<double>(), I[m], 1, R[m], nxt.as<double>());
                shape[m] = R[m];
                cur = std::move(nxt);
                src = cur.get();
                src_f32 = false;
            }
            sumsq(ctx, cur.get(), DT_F64, prod(R, N), scal.as<double>() + 2);
        }
        const double *gsrc = cur.as<double>();
        const int gslot = 2;
        DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
        // The outputs are copied (host or device, straight from the plan's
        // buffers) before the one synchronisation that reads ||X||^2 and
        // ||G||^2, the kernels' error word and the device loop's sweep count
        // and residuals (all into the context's pinned block).
        {
            void *dst[kMaxCopyBlocks];
            const void *src[kMaxCopyBlocks];
            size_t bytes[kMaxCopyBlocks];
            dst[0] = G_user;
            src[0] = gsrc;
            bytes[0] = prod(R, N) * sizeof(double);
            for (int m = 0; m < N; m++) {
                dst[1 + m] = U_user ? U_user[m] : nullptr;
                src[1 + m] = U[m].get();
                bytes[1 + m] = I[m] * R[m] * sizeof(double);
            }
            copy_blocks(ctx, 1 + N, dst, src, bytes);
        }
        constexpr size_t kErrAt = 32, kLoopAt = 64;
        static_assert(kLoopAt + sizeof(LoopState) <= dt_ctx::kHostStageBytes, "stage too small");
        char *st = static_cast<char *>(host_stage(ctx));
        DT_CUDA(cudaMemcpyAsync(st, scal.as<double>(), (gslot + 1) * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaMemcpyAsync(st + kErrAt, err.get(), sizeof(int), cudaMemcpyDeviceToHost,
                                ctx->stream));
        if (device_loop)
            DT_CUDA(cudaMemcpyAsync(st + kLoopAt, loopst.get(), sizeof(LoopState),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        double sc[gslot + 1];
        std::memcpy(sc, st, sizeof(sc));
        const double g2 = sc[gslot];
        int herr = 0;
        std::memcpy(&herr, st + kErrAt, sizeof(int));
        if (device_loop) {
            LoopState hst;
            std::memcpy(&hst, st + kLoopAt, sizeof(LoopState));
            x2 = sc[0];
            sweeps = hst.it;
            ctx->launches += (int64_t)sweeps * loop->launches_per_sweep;
            if (rep)
                for (int i = 0; i < std::min(sweeps, DT_MAX_HIST); i++) rep->res_hist[i] = hst.hist[i];
        }
        // The FP32 copy of an FP64 X lives for this call only.
        X32own.release();
        X32 = nullptr;
        if (herr) fail(DT_ERR_TIMEOUT, fmt("tensor-core kernel reported error %d (wait timed out)", herr));
        float ms = 0.f;
        DT_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        if (!std::isfinite(g2)) fail(DT_ERR_NUMERIC, "HOOI produced a non-finite core");
        if (rep) {
            rep->sweeps = sweeps;
            rep->x_norm = std::sqrt(x2);
            rep->g_norm = std::sqrt(g2);
            rep->residual = std::sqrt(std::max(0.0, 1.0 - g2 / x2));
            rep->device_ms = ms;
            rep->kernel_launches = (int)(ctx->launches - launches0);
            rep->precision_used = opts.precision;
            rep->ttm_x_launches = timer.count();
            rep->ttm_x_ms = timer.total_ms();
            rep->ttm_x_bytes = timer.bytes();
        }
        xtimer = nullptr;
    }
};

// The mixed driver's buffers and captured sweeps (one graph per precision).
struct MixedPlan {
    int N, inner, precision;
    int64_t I[16], R[16];
    MixedHooi h;
    SweepGraph g_bf16, g_split;
    LoopGraph loop;  // destroyed before h's buffers
    MixedPlan(int n, const int64_t *shape, const int64_t *ranks, const dt_hooi_opts &o)
        : N(n), inner(o.inner_iters), precision(o.precision) {
        for (int m = 0; m < n; m++) {
            I[m] = shape[m];
            R[m] = ranks[m];
        }
    }
    bool matches(int n, const int64_t *shape, const int64_t *ranks, const dt_hooi_opts &o) const {
        if (n != N || o.inner_iters != inner || o.precision != precision) return false;
        for (int m = 0; m < n; m++)
            if (shape[m] != I[m] || ranks[m] != R[m]) return false;
        return true;
    }
};

}  // namespace

bool hooi_lowprec_tc_ok(int ndim, const int64_t *shape, const int64_t *ranks) {
    return MixedHooi::plan_ok_for(ndim, shape, ranks);
}

void hooi_dense_lowprec(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
                        const int64_t *ranks, const dt_hooi_opts &opts, double *G,
                        double *const *U, dt_hooi_report *report, ChunkedUpload *upload) {
    DT_CHECK_ARG(opts.precision == DT_PREC_BF16 || opts.precision == DT_PREC_BF16X2 ||
                     opts.precision == DT_PREC_BF16XH,
                 "unknown precision %d", opts.precision);
    DT_CHECK_ARG(opts.init != DT_INIT_HOSVD,
                 "the tensor-core HOOI starts from random or given factors, not HOSVD");
    if (!MixedHooi::plan_ok_for(ndim, shape, ranks)) {
        // A shape outside the TMA / UMMA layout rules: run the FP64 engine.
        dt_hooi_opts o = opts;
        o.precision = DT_PREC_FP64;
        DenseHooi f;
        f.setup(ctx, X, dtype, ndim, shape, ranks, o);
        f.run(G, U, report);
        if (report) report->precision_used = DT_PREC_FP64;
        return;
    }
    // The plan (buffers + captured sweeps) is kept on the context for the next
    // call with the same shapes, ranks and inner iterations.
    auto plan = std::static_pointer_cast<MixedPlan>(ctx->hooi_plan_mixed);
    if (!plan || !plan->matches(ndim, shape, ranks, opts)) {
        release_plan(ctx, ctx->hooi_plan_mixed);
        plan = std::make_shared<MixedPlan>(ndim, shape, ranks, opts);
        MixedHooi &h = plan->h;
        h.ctx = ctx;
        h.N = ndim;
        for (int m = 0; m < ndim; m++) {
            h.I[m] = shape[m];
            h.R[m] = ranks[m];
        }
        h.xsize = prod(shape, ndim);
        h.U.resize(ndim);
        int64_t maxI = 0, maxR = 0;
        for (int m = 0; m < ndim; m++) {
            h.U[m].alloc(ctx, shape[m] * ranks[m] * sizeof(double));
            maxI = std::max(maxI, shape[m]);
            maxR = std::max(maxR, ranks[m]);
        }
        h.S.alloc(ctx, maxI * maxI * sizeof(double));
        h.work.alloc(ctx, (3 * maxI * maxR + maxR + 64) * sizeof(double));
        h.flag.alloc(ctx, sizeof(int));
        h.err.alloc(ctx, sizeof(int));
        h.scal.alloc(ctx, 4 * sizeof(double));
        h.Gs.alloc(ctx, prod(ranks, ndim) * sizeof(double));
        h.g_bf16 = &plan->g_bf16;
        h.g_split = &plan->g_split;
        h.loop = &plan->loop;
        h.opts = opts;
        h.xsplit = opts.precision == DT_PREC_BF16X2 ||
                   (opts.precision == DT_PREC_BF16 && opts.refine_sweeps > 0);
        h.size_arena();
        ctx->hooi_plan_mixed = plan;
    }
    MixedHooi &h = plan->h;
    h.opts = opts;
    h.X32 = nullptr;
    h.helper.setup(ctx, X, dtype, ndim, shape, ranks, opts);
    DT_CUDA(cudaMemsetAsync(h.flag.get(), 0, sizeof(int), ctx->stream));
    DT_CUDA(cudaMemsetAsync(h.err.get(), 0, sizeof(int), ctx->stream));
    h.run(X, dtype, G, U, report, upload);
}

}  // namespace dt
