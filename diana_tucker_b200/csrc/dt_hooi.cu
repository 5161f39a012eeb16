// Dense HOOI driver: Algorithm::Tucker::HOOI_ALS
// (template/algorithm/tucker/hooi_als.tpp:64-123) on one GPU.
//
// Per sweep the reference copies A and runs the full TTM chain for every mode
// (hooi_als.tpp:96-101), then recomputes the core from A (:105-109).  Here the
// chains share work through a dimension tree: the node owning modes [lo, hi)
// holds T = X x_{m not in [lo,hi)} U_m^T; its children contract the other half,
// so X itself is read twice per sweep whatever N is.  The core of a sweep is
// G = Y_{N-1} x_{N-1} U_{N-1}^T, the last leaf's chain output contracted once
// more -- the same tensor as the reference's recomputation.  The leading
// subspace of Y_(n) Y_(n)^T (ALS_, hooi_als.tpp:7-34: five subspace-iteration
// steps from the previous U_n) runs on the device from the Gram.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "dt_hooi.cuh"
#include "dt_kernels.cuh"

namespace dt {

namespace {

}  // namespace

// The sequence rand() returns after srand(seed) in the GNU C library, which
// the reference's Util::randn draws from: its additive lagged-Fibonacci
// generator of degree 31 and separation 3 (random(3), TYPE_3), restated.  The
// 31-word state is filled by the Lehmer generator x <- 16807 x mod (2^31 - 1)
// from the seed (0 taken as 1); each step adds the word 31 back to the word 3
// back (mod 2^32) and returns the sum without its lowest bit; the first 310
// steps are discarded.  Used for an explicit seed, it gives the library's own
// draws without touching the process's rand() state.
LibcRand::LibcRand(unsigned seed) {
    int32_t word = (int32_t)(seed ? seed : 1u);
    s_[0] = word;
    for (int i = 1; i < 31; i++) {
        const int64_t hi = word / 127773, lo = word % 127773;
        int64_t w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        word = (int32_t)w;
        s_[i] = word;
    }
    f_ = 3;
    r_ = 0;
    for (int i = 0; i < 310; i++) next();
}

int32_t LibcRand::next() {
    const uint32_t v = (uint32_t)s_[f_] + (uint32_t)s_[r_];
    s_[f_] = (int32_t)v;
    f_ = f_ == 30 ? 0 : f_ + 1;
    r_ = r_ == 30 ? 0 : r_ + 1;
    return (int32_t)(v >> 1);
}

namespace {

// Marsaglia polar draw on a rand()-like source -- the method of the
// reference's Util::randn (src/util.cpp:10-18), kept identical so
// DT_INIT_RANDN_LIBC starts from the reference's factors.  `gen` is the
// library's restatement of the C library's generator (explicit seed) or
// null for the process's own rand() (DT_SEED_KEEP).
double libc_polar_randn(LibcRand *gen) {
    constexpr double kRandMax = 2147483647.0;  // RAND_MAX of the GNU C library
    for (;;) {
        const double u = ((double)(gen ? gen->next() : rand()) / kRandMax) * 2 - 1;
        const double v = ((double)(gen ? gen->next() : rand()) / kRandMax) * 2 - 1;
        const double r = u * u + v * v;
        if (r == 0 || r > 1) continue;
        return u * std::sqrt(-2 * std::log(r) / r);
    }
}

// Deterministic N(0,1) for HOSVD's subspace-iteration start (splitmix64 +
// Box-Muller).
std::vector<double> seeded_gaussian(size_t n, uint64_t seed) {
    std::vector<double> out(n);
    uint64_t s = seed * 0x9E3779B97F4A7C15ULL + 0x1234567ULL;
    auto next = [&]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    for (size_t i = 0; i < n; i += 2) {
        const double u1 = ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        const double u2 = ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        const double rad = std::sqrt(-2.0 * std::log(u1));
        out[i] = rad * std::cos(6.283185307179586 * u2);
        if (i + 1 < n) out[i + 1] = rad * std::sin(6.283185307179586 * u2);
    }
    return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// FP64 engine
// ---------------------------------------------------------------------------
void DenseHooi::setup(dt_ctx *c, const void *X, int dt, int n, const int64_t *shp,
                      const int64_t *rk, const dt_hooi_opts &o) {
    ctx = c;
    dtype = dt;
    N = n;
    opts = o;
    for (int m = 0; m < N; m++) {
        I[m] = shp[m];
        R[m] = rk[m];
    }
    xsize = prod(I, N);
    Xdev = X;
    if (!allocated) {
        U.resize(N);
        for (int m = 0; m < N; m++) U[m].alloc(ctx, I[m] * R[m] * sizeof(double));
        int64_t maxI = 0, maxR = 0;
        for (int m = 0; m < N; m++) {
            maxI = std::max(maxI, I[m]);
            maxR = std::max(maxR, R[m]);
        }
        S.alloc(ctx, maxI * maxI * sizeof(double));
        work.alloc(ctx, (3 * maxI * maxR + maxR + 64) * sizeof(double));
        flag.alloc(ctx, sizeof(int));
        scal.alloc(ctx, 4 * sizeof(double));
        G.alloc(ctx, prod(R, N) * sizeof(double));
        allocated = true;
    }
    DT_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), ctx->stream));
    if (dtype == DT_F32 && N == 1) {
        if (!X64.get()) X64.alloc(ctx, xsize * sizeof(double));
        f32_to_f64(ctx, static_cast<const float *>(X), xsize, X64.as<double>());
        Xdev = X64.get();
        dtype = DT_F64;
    }
}

// Contract `t` (shape `shape`) over mode m with U_m^T into a new buffer.
DevMem DenseHooi::contract(const void *t, int tdtype, int64_t *shape, int m) {
    int64_t L = 1, B = 1;
    for (int k = 0; k < m; k++) L *= shape[k];
    for (int k = m + 1; k < N; k++) B *= shape[k];
    DevMem out(ctx, L * R[m] * B * sizeof(double));
    const bool from_x = xtimer && t == Xdev;
    if (from_x) xtimer->begin();
    if (tdtype == DT_F32)
        ttm_f64<float>(ctx, static_cast<const float *>(t), L, shape[m], B, U[m].as<double>(),
                       I[m], 1, R[m], out.as<double>());
    else
        ttm_f64<double>(ctx, static_cast<const double *>(t), L, shape[m], B,
                        U[m].as<double>(), I[m], 1, R[m], out.as<double>());
    if (from_x)
        xtimer->end((double)L * shape[m] * B * (tdtype == DT_F32 ? 4 : 8) +
                    (double)L * R[m] * B * 8 + (double)I[m] * R[m] * 8);
    shape[m] = R[m];
    return out;
}

// Contract the modes in `modes` (largest size reduction first).
DevMem DenseHooi::contract_all(const void *t, int tdtype, int64_t *shape,
                               std::vector<int> modes) {
    std::sort(modes.begin(), modes.end(), [&](int a, int b) {
        return (double)I[a] / R[a] > (double)I[b] / R[b];
    });
    DevMem cur;
    const void *src = t;
    int sdt = tdtype;
    for (int m : modes) {
        DevMem nxt = contract(src, sdt, shape, m);
        cur = std::move(nxt);
        src = cur.get();
        sdt = DT_F64;
    }
    return cur;
}

void DenseHooi::leaf(int n, const double *Y, const int64_t *shape) {
    int64_t L = 1, B = 1;
    for (int k = 0; k < n; k++) L *= shape[k];
    for (int k = n + 1; k < N; k++) B *= shape[k];
    ttt_f64(ctx, Y, Y, L, I[n], I[n], B, S.as<double>());
    subspace_iter(ctx, S.as<double>(), I[n], U[n].as<double>(), R[n], opts.inner_iters,
                  work.as<double>(), flag.as<int>());
    if (n == N - 1) {
        // Core of this sweep: G = Y x_{N-1} U_{N-1}^T (hooi_als.tpp:105-109).
        ttm_f64<double>(ctx, Y, L, I[n], 1, U[n].as<double>(), I[n], 1, R[n], G.as<double>());
        sumsq(ctx, G.get(), DT_F64, L * R[n], scal.as<double>() + 1);
    }
}

void DenseHooi::node(int lo, int hi, const void *T, int tdtype, const int64_t *shape) {
    if (hi - lo == 1) {
        leaf(lo, static_cast<const double *>(T), shape);
        return;
    }
    const int mid = (lo + hi) / 2;
    for (int side = 0; side < 2; side++) {
        const int clo = side == 0 ? lo : mid, chi = side == 0 ? mid : hi;
        std::vector<int> modes;
        for (int m = lo; m < hi; m++)
            if (m < clo || m >= chi) modes.push_back(m);
        int64_t cshape[16];
        std::memcpy(cshape, shape, N * sizeof(int64_t));
        DevMem child = contract_all(T, tdtype, cshape, modes);
        node(clo, chi, child.get(), DT_F64, cshape);
    }
}

void DenseHooi::sweep() {
    if (N == 1) {
        leaf(0, static_cast<const double *>(Xdev), I);
        return;
    }
    int64_t shape[16];
    std::memcpy(shape, I, N * sizeof(int64_t));
    node(0, N, Xdev, dtype, shape);
}

void DenseHooi::init_factors(double *const *U_user, double *const *dst) {
    auto out = [&](int m) { return dst ? dst[m] : U[m].as<double>(); };
    if (opts.init == DT_INIT_GIVEN) {
        DT_CHECK_ARG(U_user, "DT_INIT_GIVEN needs initial factors in U");
        for (int m = 0; m < N; m++) {
            DT_CHECK_ARG(U_user[m], "DT_INIT_GIVEN: U[%d] is NULL", m);
            DevView u(ctx, U_user[m], I[m] * R[m] * sizeof(double), true, false);
            DT_CUDA(cudaMemcpyAsync(out(m), u.ptr(), I[m] * R[m] * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
        }
        return;
    }
    if (opts.init == DT_INIT_RANDN_LIBC) {
        // hooi_als.tpp:74-81: U_rand(I_n x R_n).randn(); U_n = Q of reduced_QR.
        int64_t total = 0;
        for (int m = 0; m < N; m++) total += I[m] * R[m];
        const bool seeded = opts.seed != DT_SEED_KEEP;
        if (seeded && init_cached && init_seed == opts.seed) {
            // The same seed draws the same factors: copy the orthonormal ones
            // kept from the first call (the draws take ~0.1-0.5 ms of host time),
            // all modes in one launch.
            void *d[16];
            const void *src[16];
            size_t bytes[16];
            int64_t off = 0;
            for (int m = 0; m < N; m++) {
                d[m] = out(m);
                src[m] = init_cache.as<double>() + off;
                bytes[m] = I[m] * R[m] * sizeof(double);
                off += I[m] * R[m];
            }
            copy_blocks(ctx, N, d, src, bytes);
            return;
        }
        // Draw every block in mode order (the reference's order), upload once,
        // then one batched orthonormalisation launch for all modes (any
        // orthonormal basis of span(U_rand) gives the same sweeps: the TTM
        // chain's Gram matrices only see U U^T).
        LibcRand gen(seeded ? opts.seed : 1u);
        std::vector<double> h((size_t)total);
        for (auto &v : h) v = libc_polar_randn(seeded ? &gen : nullptr);
        DevMem a(ctx, total * sizeof(double));
        DT_CUDA(cudaMemcpyAsync(a.get(), h.data(), total * sizeof(double), cudaMemcpyHostToDevice,
                                ctx->stream));
        std::vector<const double *> ap(N);
        std::vector<double *> qp(N);
        int64_t off = 0;
        for (int m = 0; m < N; m++) {
            ap[m] = a.as<double>() + off;
            qp[m] = out(m);
            off += I[m] * R[m];
        }
        orth_batch(ctx, N, ap.data(), qp.data(), I, R);
        if (seeded) {
            if (!init_cache.get()) init_cache.alloc(ctx, total * sizeof(double));
            off = 0;
            for (int m = 0; m < N; m++) {
                DT_CUDA(cudaMemcpyAsync(init_cache.as<double>() + off, out(m),
                                        I[m] * R[m] * sizeof(double), cudaMemcpyDeviceToDevice,
                                        ctx->stream));
                off += I[m] * R[m];
            }
            init_cached = true;
            init_seed = opts.seed;
        }
        return;
    }
    // HOSVD: leading R_n eigenvectors of X_(n) X_(n)^T by subspace iteration
    // from a seeded Gaussian start.
    const double *X64p = static_cast<const double *>(Xdev);
    DevMem xconv;
    if (dtype == DT_F32) {
        xconv.alloc(ctx, xsize * sizeof(double));
        f32_to_f64(ctx, static_cast<const float *>(Xdev), xsize, xconv.as<double>());
        X64p = xconv.as<double>();
    }
    for (int m = 0; m < N; m++) {
        int64_t L = 1, B = 1;
        for (int k = 0; k < m; k++) L *= I[k];
        for (int k = m + 1; k < N; k++) B *= I[k];
        ttt_f64(ctx, X64p, X64p, L, I[m], I[m], B, S.as<double>());
        std::vector<double> h = seeded_gaussian((size_t)(I[m] * R[m]), 1000 + m);
        DT_CUDA(cudaMemcpyAsync(U[m].get(), h.data(), h.size() * sizeof(double),
                                cudaMemcpyHostToDevice, ctx->stream));
        subspace_iter(ctx, S.as<double>(), I[m], U[m].as<double>(), R[m], hosvd_iters,
                      work.as<double>(), flag.as<int>());
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (dst)
            DT_CUDA(cudaMemcpyAsync(dst[m], U[m].get(), I[m] * R[m] * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
    }
}

// The two passes over X of a sweep: each half of the dimension tree first
// contracts X over its largest size reduction.
double DenseHooi::x_pass_flop() const {
    if (N == 1) return 2.0 * xsize * I[0];
    double f = 0.0;
    for (int side = 0; side < 2; side++) {
        const int lo = side == 0 ? N / 2 : 0, hi = side == 0 ? N : N / 2;
        int best = lo;
        for (int m = lo; m < hi; m++)
            if ((double)I[m] / R[m] > (double)I[best] / R[best]) best = m;
        f += 2.0 * xsize * R[best];
    }
    return f;
}

double DenseHooi::x_pass_bytes() const {
    return 2.0 * xsize * (dtype == DT_F64 ? 8 : 4);
}

// Through the context's pinned block: an asynchronous copy and one
// synchronisation.
void DenseHooi::read_scalars(int k, int n, double *out) {
    double *st = static_cast<double *>(host_stage(ctx));
    DT_CUDA(cudaMemcpyAsync(st, scal.as<double>() + k, n * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, st, n * sizeof(double));
}

double DenseHooi::read_scalar(int k) {
    double h = 0.0;
    read_scalars(k, 1, &h);
    return h;
}

void DenseHooi::run(double *G_user, double *const *U_user, dt_hooi_report *rep,
                    SweepGraph *graph) {
    const int64_t launches0 = ctx->launches;
    LaunchTimer timer(ctx, opts.profile != 0);
    xtimer = &timer;
    DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
    sumsq(ctx, Xdev, dtype, xsize, scal.as<double>());
    init_factors(U_user);
    // ||X||^2 is read with the first sweep's ||G||^2 (one synchronisation).
    double x2 = -1.0;
    double prev = -1.0, res = 0.0;
    int sweeps = 0;
    for (int it = 0; it < opts.max_sweeps; it++) {
        {
            // Counted work: the sweep's two passes over X (the first
            // contraction of each half of the dimension tree).
            SummaryScope sc(ctx, "HOOI sweep (FP64)", x_pass_flop(), x_pass_bytes());
            if (graph && !opts.profile)
                graph->run(ctx, [&] { sweep(); });
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
            fprintf(stderr, "[dt_hooi] sweep %d  ||G|| = %.12e  residual = %.12e\n", it + 1,
                    std::sqrt(g2), res);
        if (opts.tol > 0 && prev >= 0 && std::fabs(res - prev) < opts.tol) break;
        prev = res;
    }
    if (x2 < 0.0) x2 = read_scalar(0);
    if (sweeps == 0) {
        // No sweep requested: the core of the initial factors.
        int64_t shape[16];
        std::memcpy(shape, I, N * sizeof(int64_t));
        std::vector<int> all(N);
        std::iota(all.begin(), all.end(), 0);
        DevMem g0 = contract_all(Xdev, dtype, shape, all);
        DT_CUDA(cudaMemcpyAsync(G.get(), g0.get(), prod(R, N) * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        sumsq(ctx, G.get(), DT_F64, prod(R, N), scal.as<double>() + 1);
    }
    DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
    // The outputs go straight from the plan's buffers into the caller's (host
    // or device), queued with the read-back of ||G||^2: one synchronisation.
    {
        void *dst[kMaxCopyBlocks];
        const void *src[kMaxCopyBlocks];
        size_t bytes[kMaxCopyBlocks];
        dst[0] = G_user;
        src[0] = G.get();
        bytes[0] = prod(R, N) * sizeof(double);
        for (int m = 0; m < N; m++) {
            dst[1 + m] = U_user ? U_user[m] : nullptr;
            src[1 + m] = U[m].get();
            bytes[1 + m] = I[m] * R[m] * sizeof(double);
        }
        copy_blocks(ctx, 1 + N, dst, src, bytes);
    }
    const double g2 = read_scalar(1);
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
        rep->precision_used = DT_PREC_FP64;
        rep->ttm_x_launches = timer.count();
        rep->ttm_x_ms = timer.total_ms();
        rep->ttm_x_bytes = timer.bytes();
    }
    xtimer = nullptr;
}

// The FP64 driver's buffers and sweep graph, kept on the context for the next
// call with the same X, shapes, ranks and inner iterations.
struct Fp64Plan {
    const void *X;
    int dtype, N, inner;
    int64_t I[16], R[16];
    DenseHooi h;
    SweepGraph graph;
    Fp64Plan(const void *x, int dt, int n, const int64_t *shape, const int64_t *ranks,
             const dt_hooi_opts &o)
        : X(x), dtype(dt), N(n), inner(o.inner_iters) {
        for (int m = 0; m < n; m++) {
            I[m] = shape[m];
            R[m] = ranks[m];
        }
    }
    bool matches(const void *x, int dt, int n, const int64_t *shape, const int64_t *ranks,
                 const dt_hooi_opts &o) const {
        if (x != X || dt != dtype || n != N || o.inner_iters != inner) return false;
        for (int m = 0; m < n; m++)
            if (shape[m] != I[m] || ranks[m] != R[m]) return false;
        return true;
    }
};

}  // namespace dt

using namespace dt;

extern "C" {

int dt_libc_rand_sequence(unsigned seed, int64_t n, int32_t *out) {
    return guard([&] {
        DT_CHECK_ARG(n >= 0 && (n == 0 || out), "dt_libc_rand_sequence: bad arguments");
        LibcRand g(seed);
        for (int64_t i = 0; i < n; i++) out[i] = g.next();
    });
}

void dt_hooi_default_opts(dt_hooi_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->init = DT_INIT_RANDN_LIBC;
    o->seed = 1;
    o->max_sweeps = 5;
    o->tol = 0.0;
    o->inner_iters = 5;
    o->precision = DT_PREC_FP64;
    o->refine_sweeps = 0;
    o->verbose = 0;
}

int dt_hooi_dense(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
                  const int64_t *ranks, const dt_hooi_opts *opts, double *G,
                  double *const *U, dt_hooi_report *report) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(X && shape && ranks, "dt_hooi_dense: null argument");
        DT_CHECK_ARG(ndim >= 1 && ndim <= 16, "dt_hooi_dense: ndim %d out of range", ndim);
        DT_CHECK_ARG(dtype == DT_F64 || dtype == DT_F32, "dt_hooi_dense: bad dtype %d", dtype);
        for (int m = 0; m < ndim; m++)
            DT_CHECK_ARG(shape[m] >= 1 && ranks[m] >= 1 && ranks[m] <= shape[m],
                         "dt_hooi_dense: need 1 <= R_%d <= I_%d (R=%lld, I=%lld)", m, m,
                         (long long)ranks[m], (long long)shape[m]);
        dt_hooi_opts o;
        if (opts)
            o = *opts;
        else
            dt_hooi_default_opts(&o);
        DT_CHECK_ARG(o.max_sweeps >= 0, "dt_hooi_dense: max_sweeps must be >= 0");
        DT_CHECK_ARG(o.inner_iters >= 1, "dt_hooi_dense: inner_iters must be >= 1");
        DT_CUDA(cudaSetDevice(ctx->device));
        if (report) std::memset(report, 0, sizeof(*report));
        const size_t esz = dtype == DT_F64 ? 8 : 4;
        // A host FP32 X of the tensor-core path is copied in chunks, all
        // issued here, before any set-up; that path rounds each chunk to BF16
        // as it lands.  Any other host X is staged in one copy.
        const bool x_host = o.precision != DT_PREC_FP64 && dtype == DT_F32 && !is_device_ptr(X) &&
                            hooi_lowprec_tc_ok(ndim, shape, ranks);
        ChunkedUpload up;
        if (x_host) up.start(ctx, X, prod(shape, ndim), sizeof(float));
        DevView x(ctx, x_host ? nullptr : X, x_host ? 0 : prod(shape, ndim) * esz, true, false);
        SummaryScope sc(ctx, "Algorithm::Tucker::HOOI_ALS()");
        if (o.precision == DT_PREC_FP64) {
            // A staged host X lives only for this call: its plan is not kept
            // and its sweeps are launched directly.
            const bool keep = x.ptr() == X;
            auto plan = std::static_pointer_cast<Fp64Plan>(ctx->hooi_plan_fp64);
            if (!keep || !plan || !plan->matches(x.ptr(), dtype, ndim, shape, ranks, o)) {
                if (keep) release_plan(ctx, ctx->hooi_plan_fp64);
                plan = std::make_shared<Fp64Plan>(x.ptr(), dtype, ndim, shape, ranks, o);
                if (keep) ctx->hooi_plan_fp64 = plan;
            }
            plan->h.setup(ctx, x.ptr(), dtype, ndim, shape, ranks, o);
            plan->h.run(G, U, report, keep ? &plan->graph : nullptr);
        } else {
            hooi_dense_lowprec(ctx, x_host ? up.dst.get() : x.ptr(), dtype, ndim, shape, ranks, o,
                               G, U, report, x_host ? &up : nullptr);
        }
    });
}

}  // extern "C"
