// .tns ingest on the device: replaces read_data<double> (src/read_data.cpp:
// 36-129), which parses the text on one host thread.
//
//  1. The bytes go to the device once.
//  2. Line starts: each CTA counts the newlines of its 64 KB chunk; an
//     exclusive scan of the counts gives every chunk its first line; a second
//     pass writes the offset after each newline (a block scan orders them).
//  3. One thread per line splits it into whitespace-separated tokens: ndim
//     1-based indices, then the value.  Blank lines are skipped (compacted
//     out); a malformed line fails the call with its line number.
//  4. dims = max index + 1 per mode (read_data.cpp:117-126).
//
// Values: sign, digits, '.', digits, exponent.  At most 19 significant digits
// are kept as an integer M with a decimal exponent e.  M <= 2^53 and |e| <= 22
// is exact in one IEEE operation (Clinger's fast path); otherwise M * 10^e is
// formed in double-double arithmetic (Dekker's two-product, relative error
// ~2^-100) and rounded once, which is the correctly rounded result unless the
// decimal value lies within that error of a halfway point between doubles.
// Results in the subnormal range (below 2.2e-308) may be one unit off.
#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dt_core.cuh"

namespace dt {
namespace {

constexpr int TNS_MAXD = 8;
constexpr int64_t TNS_CHUNK = 64 * 1024;  // bytes per CTA in the newline scan
constexpr int TNS_THREADS = 256;
constexpr int TNS_PER_THREAD = (int)(TNS_CHUNK / TNS_THREADS);

enum : int { LINE_OK = 0, LINE_BLANK = 1, LINE_BAD_TOKENS = 2, LINE_BAD_NUMBER = 3, LINE_BAD_INDEX = 4 };

__global__ void count_newlines_kernel(const char *__restrict__ buf, int64_t size,
                                      int64_t *__restrict__ counts) {
    const int64_t c0 = blockIdx.x * TNS_CHUNK + (int64_t)threadIdx.x * TNS_PER_THREAD;
    int n = 0;
    for (int j = 0; j < TNS_PER_THREAD; j++) {
        const int64_t p = c0 + j;
        if (p < size && buf[p] == '\n') n++;
    }
    using BR = cub::BlockReduce<int, TNS_THREADS>;
    __shared__ typename BR::TempStorage tmp;
    const int total = BR(tmp).Sum(n);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// starts[0] = 0; starts[k] = (offset of the k-th newline) + 1.
__global__ void write_starts_kernel(const char *__restrict__ buf, int64_t size,
                                    const int64_t *__restrict__ first,
                                    int64_t *__restrict__ starts) {
    const int64_t c0 = blockIdx.x * TNS_CHUNK + (int64_t)threadIdx.x * TNS_PER_THREAD;
    int n = 0;
    for (int j = 0; j < TNS_PER_THREAD; j++) {
        const int64_t p = c0 + j;
        if (p < size && buf[p] == '\n') n++;
    }
    using BS = cub::BlockScan<int, TNS_THREADS>;
    __shared__ typename BS::TempStorage tmp;
    int before = 0;
    BS(tmp).ExclusiveSum(n, before);
    int64_t k = first[blockIdx.x] + before;
    for (int j = 0; j < TNS_PER_THREAD && n > 0; j++) {
        const int64_t p = c0 + j;
        if (p < size && buf[p] == '\n') {
            starts[k + 1] = p + 1;
            k++;
            n--;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = 0;
}

// ---- double-double helpers (Dekker / Knuth error-free transformations) ----
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ DD dd_norm(double hi, double lo) {
    const double s = hi + lo;
    return {s, lo - (s - hi)};
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = a.hi * b.hi;
    if (isinf(p)) return {p, 0.0};
    const double e = fma(a.hi, b.hi, -p);
    return dd_norm(p, e + (a.hi * b.lo + a.lo * b.hi));
}
__device__ __forceinline__ DD dd_mul_d(DD a, double b) {
    const double p = a.hi * b;
    if (isinf(p)) return {p, 0.0};
    const double e = fma(a.hi, b, -p);
    return dd_norm(p, e + a.lo * b);
}
__device__ __forceinline__ DD dd_sub(DD a, DD b) {
    const DD s = dd_two_sum(a.hi, -b.hi);
    return dd_norm(s.hi, s.lo + (a.lo - b.lo));
}
__device__ __forceinline__ DD dd_div(DD a, DD b) {
    const double q1 = a.hi / b.hi;
    DD r = dd_sub(a, dd_mul_d(b, q1));
    const double q2 = r.hi / b.hi;
    r = dd_sub(r, dd_mul_d(b, q2));
    const double q3 = r.hi / b.hi;
    const DD q = dd_norm(q1, q2);
    return dd_norm(q.hi, q.lo + q3);
}

// 10^k, k in [0, 22]: every one is an exact double.
__device__ __forceinline__ double pow10_exact(int k) {
    double p = 1.0;
    for (int i = 0; i < k; i++) p *= 10.0;
    return p;
}

// 10^n (n >= 0) in double-double: powers of 10^22 (exact) times an exact
// remainder.
__device__ DD dd_pow10(int n) {
    DD r = {pow10_exact(n % 22), 0.0};
    const DD big = {pow10_exact(22), 0.0};
    for (int q = n / 22; q > 0; q--) r = dd_mul(r, big);
    return r;
}

__device__ __forceinline__ bool is_digit(char c) { return c >= '0' && c <= '9'; }
__device__ __forceinline__ bool is_space(char c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\n';
}

// [s, e) holds one token.
__device__ bool parse_double(const char *s, const char *e, double *out) {
    bool neg = false;
    if (s < e && (*s == '+' || *s == '-')) {
        neg = *s == '-';
        s++;
    }
    uint64_t M = 0;
    int nd = 0, ex = 0;
    bool any = false;
    while (s < e && is_digit(*s)) {
        const int d = *s - '0';
        any = true;
        if (M == 0 && d == 0) {
        } else if (nd < 19) {
            M = M * 10 + d;
            nd++;
        } else {
            ex++;
        }
        s++;
    }
    if (s < e && *s == '.') {
        s++;
        while (s < e && is_digit(*s)) {
            const int d = *s - '0';
            any = true;
            if (M == 0 && d == 0) {
                ex--;
            } else if (nd < 19) {
                M = M * 10 + d;
                nd++;
                ex--;
            }
            s++;
        }
    }
    if (!any) return false;
    if (s < e && (*s == 'e' || *s == 'E')) {
        s++;
        bool eneg = false;
        if (s < e && (*s == '+' || *s == '-')) {
            eneg = *s == '-';
            s++;
        }
        if (s >= e || !is_digit(*s)) return false;
        int x = 0;
        while (s < e && is_digit(*s)) {
            if (x < 100000) x = x * 10 + (*s - '0');
            s++;
        }
        ex += eneg ? -x : x;
    }
    if (s != e) return false;
    double v;
    if (M == 0) {
        v = 0.0;
    } else if (M <= (uint64_t(1) << 53) && ex >= -22 && ex <= 22) {
        v = (double)M;
        v = ex < 0 ? v / pow10_exact(-ex) : v * pow10_exact(ex);
    } else if (ex > 308 + 19) {
        v = INFINITY;
    } else if (ex < -342 - 19) {
        v = 0.0;
    } else {
        const double mh = (double)M;
        const DD m = {mh, (double)(int64_t)(M - (uint64_t)mh)};
        // Two double-double scalings (|e1| <= 270 keeps M 10^e1 and 10^|e2|
        // finite), then one rounding.
        int e1 = ex, e2 = 0;
        if (e1 > 270) {
            e2 = e1 - 270;
            e1 = 270;
        } else if (e1 < -270) {
            e2 = e1 + 270;
            e1 = -270;
        }
        DD r = e1 >= 0 ? dd_mul(m, dd_pow10(e1)) : dd_div(m, dd_pow10(-e1));
        if (e2 > 0) r = dd_mul(r, dd_pow10(e2));
        if (e2 < 0) r = dd_div(r, dd_pow10(-e2));
        v = r.hi + r.lo;
    }
    *out = neg ? -v : v;
    return true;
}

__device__ bool parse_index(const char *s, const char *e, int64_t *out) {
    if (s < e && *s == '+') s++;
    if (s >= e) return false;
    int64_t v = 0;
    while (s < e) {
        if (!is_digit(*s)) return false;
        if (v > (int64_t(1) << 58)) return false;
        v = v * 10 + (*s - '0');
        s++;
    }
    *out = v;
    return true;
}

// One thread per line: ndim indices (1-based in the file, 0-based out) and a
// value; status[k] says what the line was.
__global__ void parse_lines_kernel(const char *__restrict__ buf, int64_t size,
                                   const int64_t *__restrict__ starts, int64_t nlines, int ndim,
                                   int64_t *__restrict__ idx, double *__restrict__ vals,
                                   int *__restrict__ status) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nlines;
         k += (int64_t)gridDim.x * blockDim.x) {
        const char *const b0 = buf + starts[k];
        const char *end = buf + (k + 1 < nlines ? starts[k + 1] - 1 : size);
        // Token count first, so a short or long line is reported as such.
        int tok = 0;
        for (const char *p = b0; p < end;) {
            while (p < end && is_space(*p)) p++;
            if (p >= end) break;
            while (p < end && !is_space(*p)) p++;
            tok++;
        }
        int st = tok == 0 ? LINE_BLANK : tok != ndim + 1 ? LINE_BAD_TOKENS : LINE_OK;
        const char *p = b0;
        for (int t = 0; st == LINE_OK && t <= ndim; t++) {
            while (p < end && is_space(*p)) p++;
            const char *t0 = p;
            while (p < end && !is_space(*p)) p++;
            if (t < ndim) {
                int64_t v = 0;
                if (!parse_index(t0, p, &v))
                    st = LINE_BAD_NUMBER;
                else if (v < 1)
                    st = LINE_BAD_INDEX;
                else
                    idx[(int64_t)t * nlines + k] = v - 1;
            } else {
                double v = 0.0;
                if (!parse_double(t0, p, &v))
                    st = LINE_BAD_NUMBER;
                else
                    vals[k] = v;
            }
        }
        status[k] = st;
    }
}

// keep[k] = status is OK; bad = smallest line number with a parse error.
__global__ void line_flags_kernel(const int *__restrict__ status, int64_t nlines,
                                  int *__restrict__ keep, unsigned long long *__restrict__ bad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nlines;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int s = status[k];
        keep[k] = s == LINE_OK;
        if (s >= LINE_BAD_TOKENS)
            atomicMin(bad, ((unsigned long long)k << 8) | (unsigned long long)s);
    }
}

}  // namespace
}  // namespace dt

struct dt_tns {
    dt_ctx *ctx = nullptr;
    int ndim = 0;
    int64_t nnz = 0;
    int64_t dims[dt::TNS_MAXD] = {};
    dt::DevMem idx;   // int64 [ndim][nnz]
    dt::DevMem vals;  // double [nnz]
};

using namespace dt;

namespace {

// Number of whitespace-separated tokens on the first non-blank line.
int first_line_tokens(const char *h, int64_t n) {
    int64_t p = 0;
    while (p < n) {
        int tok = 0;
        bool in = false;
        for (; p < n && h[p] != '\n'; p++) {
            const bool sp = h[p] == ' ' || h[p] == '\t' || h[p] == '\r';
            if (!sp && !in) tok++;
            in = !sp;
        }
        if (tok > 0) return tok;
        p++;
    }
    return 0;
}

dt_tns *parse_device(dt_ctx *ctx, const char *dbuf, int64_t size, const char *head,
                     int64_t head_n, bool head_complete) {
    int tokens = first_line_tokens(head, head_n);
    DT_CHECK_ARG(tokens > 0 || !head_complete, ".tns: no data line");
    DT_CHECK_ARG(tokens > 0, ".tns: first data line longer than %lld bytes", (long long)head_n);
    const int ndim = tokens - 1;
    SummaryScope sc(ctx, "read_data()", 0.0, (double)size);
    DT_CHECK_ARG(ndim >= 1 && ndim <= TNS_MAXD, ".tns: %d indices per line (1..%d supported)",
                 ndim, TNS_MAXD);
    const int64_t nchunks = (size + TNS_CHUNK - 1) / TNS_CHUNK;
    DevMem counts(ctx, (nchunks + 1) * sizeof(int64_t)), first(ctx, (nchunks + 1) * sizeof(int64_t));
    DT_CUDA(cudaMemsetAsync(counts.get(), 0, (nchunks + 1) * sizeof(int64_t), ctx->stream));
    DT_LAUNCH(ctx, count_newlines_kernel, (unsigned)nchunks, TNS_THREADS, 0, dbuf, size,
              counts.as<int64_t>());
    size_t tb = 0;
    DT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts.as<int64_t>(), first.as<int64_t>(),
                                          (int)(nchunks + 1), ctx->stream));
    DevMem tmp(ctx, tb);
    DT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, counts.as<int64_t>(), first.as<int64_t>(),
                                          (int)(nchunks + 1), ctx->stream));
    ctx->launches += 1;
    int64_t nl = 0;
    DT_CUDA(cudaMemcpyAsync(&nl, first.as<int64_t>() + nchunks, sizeof(int64_t),
                            cudaMemcpyDeviceToHost, ctx->stream));
    char last = '\n';
    DT_CUDA(cudaMemcpyAsync(&last, dbuf + size - 1, 1, cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    // Lines: one per newline, plus the tail after the last one when it is
    // non-empty.
    const int64_t nlines = nl + (last != '\n' ? 1 : 0);
    DT_CHECK_ARG(nlines >= 1, ".tns: no data line");
    DevMem starts(ctx, (nl + 2) * sizeof(int64_t));
    DT_LAUNCH(ctx, write_starts_kernel, (unsigned)nchunks, TNS_THREADS, 0, dbuf, size,
              first.as<int64_t>(), starts.as<int64_t>());
    DevMem idx(ctx, (size_t)ndim * nlines * sizeof(int64_t)), vals(ctx, nlines * sizeof(double)),
        status(ctx, nlines * sizeof(int)), keep(ctx, nlines * sizeof(int));
    const unsigned blocks =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((nlines + 255) / 256, 16 * ctx->num_sms));
    DT_LAUNCH(ctx, parse_lines_kernel, blocks, 256, 0, dbuf, size, starts.as<int64_t>(), nlines,
              ndim, idx.as<int64_t>(), vals.as<double>(), status.as<int>());
    DevMem bad(ctx, sizeof(unsigned long long));
    DT_CUDA(cudaMemsetAsync(bad.get(), 0xff, sizeof(unsigned long long), ctx->stream));
    DT_LAUNCH(ctx, line_flags_kernel, blocks, 256, 0, status.as<int>(), nlines, keep.as<int>(),
              bad.as<unsigned long long>());
    unsigned long long hbad = 0;
    DT_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(hbad), cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    if (hbad != ~0ull) {
        const long long line = (long long)(hbad >> 8) + 1;
        const int why = (int)(hbad & 0xff);
        fail(DT_ERR_ARG, fmt(".tns line %lld: %s", line,
                             why == LINE_BAD_TOKENS ? "expected ndim indices and one value"
                             : why == LINE_BAD_INDEX ? "index below 1 (indices are 1-based)"
                                                     : "not a number"));
    }
    auto *t = new dt_tns();
    try {
        t->ctx = ctx;
        t->ndim = ndim;
        // Drop blank lines (stable compaction of every mode's indices and the
        // values by the keep flags).
        DevMem nsel(ctx, sizeof(int64_t));
        size_t sb = 0;
        DT_CUDA(cub::DeviceSelect::Flagged(nullptr, sb, vals.as<double>(), keep.as<int>(),
                                           vals.as<double>(), nsel.as<int64_t>(), nlines,
                                           ctx->stream));
        DevMem stmp(ctx, sb);
        t->vals.alloc(ctx, nlines * sizeof(double));
        DT_CUDA(cub::DeviceSelect::Flagged(stmp.get(), sb, vals.as<double>(), keep.as<int>(),
                                           t->vals.as<double>(), nsel.as<int64_t>(), nlines,
                                           ctx->stream));
        t->idx.alloc(ctx, (size_t)ndim * nlines * sizeof(int64_t));
        int64_t nnz = 0;
        DT_CUDA(cudaMemcpyAsync(&nnz, nsel.get(), sizeof(int64_t), cudaMemcpyDeviceToHost,
                                ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int m = 0; m < ndim; m++) {
            DT_CUDA(cub::DeviceSelect::Flagged(stmp.get(), sb, idx.as<int64_t>() + m * nlines,
                                               keep.as<int>(),
                                               t->idx.as<int64_t>() + (int64_t)m * nnz,
                                               nsel.as<int64_t>(), nlines, ctx->stream));
        }
        ctx->launches += 1 + ndim;
        DT_CHECK_ARG(nnz >= 1, ".tns: no data line");
        t->nnz = nnz;
        // dims = max index + 1.
        DevMem mx(ctx, ndim * sizeof(int64_t));
        size_t rb = 0;
        DT_CUDA(cub::DeviceReduce::Max(nullptr, rb, t->idx.as<int64_t>(), mx.as<int64_t>(), nnz,
                                       ctx->stream));
        DevMem rtmp(ctx, rb);
        for (int m = 0; m < ndim; m++)
            DT_CUDA(cub::DeviceReduce::Max(rtmp.get(), rb, t->idx.as<int64_t>() + m * nnz,
                                           mx.as<int64_t>() + m, nnz, ctx->stream));
        ctx->launches += ndim;
        int64_t hmx[TNS_MAXD];
        DT_CUDA(cudaMemcpyAsync(hmx, mx.get(), ndim * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int m = 0; m < ndim; m++) t->dims[m] = hmx[m] + 1;
    } catch (...) {
        delete t;
        throw;
    }
    return t;
}

}  // namespace

extern "C" {

int dt_tns_parse(dt_ctx *ctx, const char *bytes, int64_t size, dt_tns **out, int *ndim,
                 int64_t *nnz) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(bytes && out && size >= 1, "dt_tns_parse: null or empty input");
        DT_CUDA(cudaSetDevice(ctx->device));
        DevView d(ctx, bytes, (size_t)size, true, false);
        std::vector<char> head((size_t)std::min<int64_t>(size, 1 << 16));
        DT_CUDA(cudaMemcpyAsync(head.data(), d.ptr(), head.size(), cudaMemcpyDefault, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        dt_tns *t = parse_device(ctx, d.as<char>(), size, head.data(), (int64_t)head.size(),
                                 (int64_t)head.size() == size);
        *out = t;
        if (ndim) *ndim = t->ndim;
        if (nnz) *nnz = t->nnz;
    });
}

int dt_tns_read(dt_ctx *ctx, const char *path, dt_tns **out, int *ndim, int64_t *nnz) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(path && out, "dt_tns_read: null argument");
        FILE *f = std::fopen(path, "rb");
        DT_CHECK_ARG(f, "dt_tns_read: cannot open %s", path);
        std::vector<char> h;
        try {
            std::fseek(f, 0, SEEK_END);
            const long n = std::ftell(f);
            std::fseek(f, 0, SEEK_SET);
            DT_CHECK_ARG(n > 0, "dt_tns_read: %s is empty", path);
            h.resize((size_t)n);
            DT_CHECK_ARG(std::fread(h.data(), 1, (size_t)n, f) == (size_t)n,
                         "dt_tns_read: short read on %s", path);
        } catch (...) {
            std::fclose(f);
            throw;
        }
        std::fclose(f);
        DT_CUDA(cudaSetDevice(ctx->device));
        DevMem d(ctx, h.size());
        DT_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size(), cudaMemcpyHostToDevice, ctx->stream));
        dt_tns *t = parse_device(ctx, d.as<char>(), (int64_t)h.size(), h.data(),
                                 (int64_t)h.size(), true);
        *out = t;
        if (ndim) *ndim = t->ndim;
        if (nnz) *nnz = t->nnz;
    });
}

int dt_tns_copy(dt_ctx *ctx, const dt_tns *t, int64_t *dims, int64_t *const *idx, double *vals) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(t && t->ctx == ctx, "dt_tns_copy: tensor of another context");
        DT_CUDA(cudaSetDevice(ctx->device));
        if (dims)
            for (int m = 0; m < t->ndim; m++) dims[m] = t->dims[m];
        if (idx)
            for (int m = 0; m < t->ndim; m++) {
                if (!idx[m]) continue;
                DT_CUDA(cudaMemcpyAsync(idx[m], t->idx.as<int64_t>() + (int64_t)m * t->nnz,
                                        t->nnz * sizeof(int64_t), cudaMemcpyDefault, ctx->stream));
            }
        if (vals)
            DT_CUDA(cudaMemcpyAsync(vals, t->vals.get(), t->nnz * sizeof(double), cudaMemcpyDefault,
                                    ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_tns_to_sptensor(dt_ctx *ctx, const dt_tns *t, dt_sptensor **sp) {
    const int64_t *ptrs[TNS_MAXD] = {};
    const int rc = guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(t && t->ctx == ctx, "dt_tns_to_sptensor: tensor of another context");
        for (int m = 0; m < t->ndim; m++) ptrs[m] = t->idx.as<int64_t>() + (int64_t)m * t->nnz;
    });
    if (rc != DT_OK) return rc;
    return dt_sptensor_create(ctx, t->nnz, t->ndim, ptrs, t->vals.as<double>(), t->dims, sp);
}

int dt_tns_destroy(dt_tns *t) {
    return guard([&] {
        if (!t) return;
        if (t->ctx) {
            cudaSetDevice(t->ctx->device);
            cudaStreamSynchronize(t->ctx->stream);
        }
        delete t;
    });
}

}  // extern "C"
