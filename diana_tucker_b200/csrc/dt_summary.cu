// Summary profiler: the reference's Summary (include/summary.hpp:27-60,
// src/summary.cpp) over CUDA events.  Library operations open named, nested
// ranges; a range records an event pair on the context's stream, and its flop
// and byte counts go to its caller when it ends (summary.cpp:48-66).  The
// table has the reference's columns: per name the total time, the share of it
// spent in nested ranges (Time C.), the count, the average time, GFlop/s and
// GB/s (summary.cpp:100-206).  Times are device times between the events.
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "dt_core.cuh"

namespace dt {

struct SummaryState {
    struct Event {
        std::string name;
        int64_t caller;
        long long flop, bytes;
        cudaEvent_t a = nullptr, b = nullptr;
        std::vector<size_t> callees;
    };
    bool on = false;
    std::vector<Event> ev;
    std::map<std::string, std::vector<size_t>> by_name;
    int64_t last = -1;

    ~SummaryState() { clear(); }
    void clear() {
        for (auto &e : ev) {
            if (e.a) cudaEventDestroy(e.a);
            if (e.b) cudaEventDestroy(e.b);
        }
        ev.clear();
        by_name.clear();
        last = -1;
    }
};

namespace {

SummaryState *state(dt_ctx *ctx) { return static_cast<SummaryState *>(ctx->summary.get()); }

void start_range(dt_ctx *ctx, const std::string &name, long long flop, long long bytes) {
    SummaryState *s = state(ctx);
    SummaryState::Event e{name, s->last, flop, bytes, nullptr, nullptr, {}};
    DT_CUDA(cudaEventCreate(&e.a));
    DT_CUDA(cudaEventCreate(&e.b));
    DT_CUDA(cudaEventRecord(e.a, ctx->stream));
    s->ev.push_back(std::move(e));
    s->last = (int64_t)s->ev.size() - 1;
    s->by_name[name].push_back((size_t)s->last);
}

void end_range(dt_ctx *ctx) {
    SummaryState *s = state(ctx);
    if (s->last < 0) return;
    const size_t i = (size_t)s->last;
    DT_CUDA(cudaEventRecord(s->ev[i].b, ctx->stream));
    s->last = s->ev[i].caller;
    if (s->last >= 0) {
        SummaryState::Event &c = s->ev[(size_t)s->last];
        c.callees.push_back(i);
        c.flop += s->ev[i].flop;
        c.bytes += s->ev[i].bytes;
    }
}

void pad(std::string &out, const std::string &d, size_t len) {
    std::string t = d;
    while (t.size() < len) t += ' ';
    out += t;
}

void rule(std::string &out, int a, int b, int c) {
    out += "|-" + std::string(a, '-') + "+-" + std::string(b, '-') + "+-" + std::string(c, '-') +
           "|\n";
}

std::string num(double v) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.6f", v);
    return b;
}

}  // namespace

bool summary_active(dt_ctx *ctx) { return ctx && ctx->summary && state(ctx)->on; }

SummaryScope::SummaryScope(dt_ctx *ctx, const char *name, double flop, double bytes) {
    if (!ctx || !ctx->summary || !state(ctx)->on) return;
    ctx_ = ctx;
    start_range(ctx, name, (long long)flop, (long long)bytes);
}

SummaryScope::~SummaryScope() {
    if (!ctx_) return;
    try {
        end_range(ctx_);
    } catch (...) {
    }
}

}  // namespace dt

using namespace dt;

extern "C" {

int dt_summary_enable(dt_ctx *ctx, int on) {
    return guard([&] {
        check_ctx(ctx);
        DT_CUDA(cudaSetDevice(ctx->device));
        if (!ctx->summary) ctx->summary = std::make_shared<SummaryState>();
        SummaryState *s = state(ctx);
        if (on && !s->on) {
            s->on = true;
            start_range(ctx, "{Main}", 0, 0);
        } else if (!on && s->on) {
            while (s->last >= 0) end_range(ctx);
            s->on = false;
        }
    });
}

int dt_summary_reset(dt_ctx *ctx) {
    return guard([&] {
        check_ctx(ctx);
        if (!ctx->summary) return;
        DT_CUDA(cudaSetDevice(ctx->device));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        SummaryState *s = state(ctx);
        s->clear();
        if (s->on) start_range(ctx, "{Main}", 0, 0);
    });
}

int dt_summary_table(dt_ctx *ctx, char *buf, int64_t size, int64_t *needed) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(buf || size == 0, "dt_summary_table: null buffer");
        DT_CUDA(cudaSetDevice(ctx->device));
        std::string out;
        if (ctx->summary) {
            SummaryState *s = state(ctx);
            // Close the open ranges ({Main} last); recording restarts below.
            const bool was_on = s->on;
            while (s->last >= 0) end_range(ctx);
            DT_CUDA(cudaStreamSynchronize(ctx->stream));
            std::vector<double> len(s->ev.size(), 0.0), counted(s->ev.size(), 0.0);
            for (size_t i = 0; i < s->ev.size(); i++) {
                float ms = 0.f;
                DT_CUDA(cudaEventElapsedTime(&ms, s->ev[i].a, s->ev[i].b));
                len[i] = ms * 1e-3;
            }
            for (size_t i = 0; i < s->ev.size(); i++)
                for (size_t c : s->ev[i].callees) counted[i] += len[c];
            const int F = 10, C = 15;
            const std::string sep = "| ";
            rule(out, F, 4 * C, 2 * C);
            out += sep;
            pad(out, "", F);
            out += sep;
            for (const char *c : {"Time(s)", "Time C.(%)", "Number", "Avg. Time(s)"}) pad(out, c, C);
            out += sep;
            for (const char *c : {"GFlop/s", "Bandw.(GB/s)"}) pad(out, c, C);
            out += sep + "\n";
            rule(out, F, 4 * C, 2 * C);
            for (const auto &kv : s->by_name) {
                double t = 0.0, tc = 0.0;
                long long flop = 0, bytes = 0;
                for (size_t i : kv.second) {
                    t += len[i];
                    tc += counted[i];
                    flop += s->ev[i].flop;
                    bytes += s->ev[i].bytes;
                }
                const double tt = t > 0 ? t : 1e-30;
                out += sep;
                pad(out, kv.first, F + 4 * C + sep.size());
                out += sep;
                if (kv.first == "{Main}") {
                    pad(out, num((double)flop / 1e9 / tt), C);
                    pad(out, num((double)bytes / 1073741824.0 / tt), C);
                } else {
                    pad(out, "", 2 * C);
                }
                out += sep + "\n" + sep;
                pad(out, "", F);
                out += sep;
                pad(out, num(t), C);
                pad(out, tc == 0.0 ? std::string("Kernel") : num(tc / tt * 100.0), C);
                pad(out, std::to_string(kv.second.size()), C);
                pad(out, num(t / (double)kv.second.size()), C);
                out += sep;
                pad(out, num((double)flop / 1e9 / tt), C);
                pad(out, num((double)bytes / 1073741824.0 / tt), C);
                out += sep + "\n";
                rule(out, F, 4 * C, 2 * C);
            }
            if (was_on) {
                s->clear();
                start_range(ctx, "{Main}", 0, 0);
            }
        }
        if (needed) *needed = (int64_t)out.size() + 1;
        if (size > 0) {
            const size_t n = std::min<size_t>(out.size(), (size_t)size - 1);
            std::memcpy(buf, out.data(), n);
            buf[n] = '\0';
        }
    });
}

}  // extern "C"
