// Shared host-side machinery of libdt_cuda.so: the context, error handling,
// host/device pointer staging and launch accounting.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <functional>
#include <memory>
#include <unordered_set>
#include <vector>

#include "dt_cuda.h"

struct dt_sptensor;

struct dt_ctx {
    // Sparse tensors created on this context; dt_ctx_destroy frees their device
    // memory and detaches them, so a later dt_sptensor_destroy only frees the
    // host object.
    std::unordered_set<dt_sptensor *> sptensors;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int num_sms = 0;
    int64_t launches = 0;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    // Device bytes held through DevMem, their maximum, and the caller's cap
    // (0: none).
    uint64_t mem_in_use = 0, mem_peak = 0, mem_limit = 0;
    // Chunked host-to-device staging: a copy stream whose chunks the context
    // stream waits for one by one (created on first use).
    static constexpr int kCopyChunks = 4;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ev[kCopyChunks + 1] = {};
    // Pinned host memory for the small read-backs (norms, residuals, error
    // words): copies into it stay asynchronous, so a call queues all of them
    // and synchronises once (allocated on first use).
    static constexpr size_t kHostStageBytes = 4096;
    void *host_stage = nullptr;
    // The dense HOOI drivers' last plans (device buffers plus a captured graph
    // of one sweep), reused by the next call with the same shapes, ranks and
    // options; released before the stream at dt_ctx_destroy.
    std::shared_ptr<void> hooi_plan_fp64, hooi_plan_mixed;
    // The batched HOOI's tuned configurations, instantiated graphs and
    // device-resident argument block (dt_hooi_batched).
    std::shared_ptr<void> batched;
    // Summary profiler state (dt_summary_*; null until first enabled).
    std::shared_ptr<void> summary;
};

namespace dt {

// Internal failures are C++ exceptions; every extern "C" entry point converts
// them into a status code plus the thread-local message of dt_last_error().
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

std::string fmt(const char *f, ...);
void set_last_error(const std::string &msg);
void clear_last_error();

[[noreturn]] inline void fail(int code, const std::string &msg) { throw Error(code, msg); }

#define DT_CHECK_ARG(cond, ...)                                            \
    do {                                                                   \
        if (!(cond)) ::dt::fail(DT_ERR_ARG, ::dt::fmt(__VA_ARGS__));       \
    } while (0)

#define DT_CUDA(expr)                                                      \
    do {                                                                   \
        cudaError_t e_ = (expr);                                           \
        if (e_ != cudaSuccess)                                             \
            ::dt::fail(e_ == cudaErrorMemoryAllocation ? DT_ERR_NOMEM      \
                                                       : DT_ERR_CUDA,      \
                       ::dt::fmt("%s failed: %s (%s:%d)", #expr,           \
                                 cudaGetErrorString(e_), __FILE__,         \
                                 __LINE__));                               \
    } while (0)

// Every kernel launch goes through this so the context can report how many
// of this library's kernels a call ran, and launch errors surface at once.
#define DT_LAUNCH(ctx, kernel, grid, block, smem, ...)                     \
    do {                                                                   \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);   \
        (ctx)->launches++;                                                 \
        DT_CUDA(cudaGetLastError());                                       \
    } while (0)

// Programmatic dependent launch.  A kernel launched with DT_LAUNCH_PDL may
// start while the previous kernel in the stream is still running: it must run
// pdl_wait() before it reads anything that kernel writes (and before it
// writes anything that kernel reads), and it may do set-up work (barriers,
// TMEM, shared-memory zeroing) before that.  pdl_trigger() lets the next
// kernel start its own set-up; every kernel of the sweep calls it early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// DT_DISABLE_PDL=1 in the environment launches these kernels in plain
// stream order (for diagnosis).
bool pdl_enabled();
// DT_DISABLE_GRAPHS=1 in the environment launches every sweep directly.
bool graphs_enabled();
// Whether the Summary profiler is recording on ctx.
bool summary_active(dt_ctx *ctx);

template <class... KArgs, class... Args>
void launch_pdl(dt_ctx *ctx, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    const bool plain_stream = ctx->stream != nullptr && ctx->stream != cudaStreamLegacy &&
                              ctx->stream != cudaStreamPerThread;
    cfg.numAttrs = pdl_enabled() && plain_stream ? 1 : 0;
    DT_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
    ctx->launches++;
}

#define DT_LAUNCH_PDL(ctx, kernel, grid, block, smem, ...) \
    ::dt::launch_pdl((ctx), (kernel), dim3(grid), dim3(block), (smem), __VA_ARGS__)

// Runs fn() and converts a thrown dt::Error into a status code.
template <class F>
int guard(F &&fn) {
    try {
        clear_last_error();
        fn();
        return DT_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return DT_ERR_NOMEM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return DT_ERR_CUDA;
    }
}

inline void check_ctx(const dt_ctx *ctx) {
    if (!ctx) fail(DT_ERR_ARG, "null dt_ctx");
}

bool is_device_ptr(const void *p);

// Validates a dense shape: 1 <= ndim <= 16, every mode >= 1, and the element
// count (so every product of modes) below 2^62.  Fails with DT_ERR_ARG naming
// `who`.
void check_shape(int ndim, const int64_t *shape, const char *who);

// Raises a kernel's dynamic shared-memory limit to at least `bytes` on ctx's
// device; the runtime is called only when the limit has to grow.
void raise_smem_limit(dt_ctx *ctx, const void *kernel, size_t bytes);
template <class K>
inline void smem_limit(dt_ctx *ctx, K *kernel, size_t bytes) {
    raise_smem_limit(ctx, reinterpret_cast<const void *>(kernel), bytes);
}

// One launch sequence (a HOOI sweep) captured as a CUDA graph and replayed on
// ctx->stream.  Capture fails over to direct execution: run() then calls fn()
// itself (the capture executed nothing).  Graphs are not used on the legacy
// or per-thread default streams, or when DT_DISABLE_GRAPHS=1.
class SweepGraph {
   public:
    SweepGraph() = default;
    SweepGraph(const SweepGraph &) = delete;
    SweepGraph &operator=(const SweepGraph &) = delete;
    ~SweepGraph() { reset(); }
    void reset();
    // Executes fn's launches: from the graph when it exists, else by capturing
    // fn into it first; falls back to calling fn directly.
    void run(dt_ctx *ctx, const std::function<void()> &fn);
    bool captured() const { return exec_ != nullptr; }

   private:
    cudaGraphExec_t exec_ = nullptr;
    int64_t launches_ = 0;
    bool failed_ = false;
};

// A named range of the Summary profiler (dt_summary_enable): CUDA events on
// ctx->stream around the scope, nested in the enclosing range, with the
// operation's flop and byte counts.  Does nothing unless the profiler is on.
// Not for use inside stream capture.
class SummaryScope {
   public:
    SummaryScope(dt_ctx *ctx, const char *name, double flop = 0, double bytes = 0);
    ~SummaryScope();
    SummaryScope(const SummaryScope &) = delete;
    SummaryScope &operator=(const SummaryScope &) = delete;

   private:
    dt_ctx *ctx_ = nullptr;
};

// Drops a cached HOOI plan once the work queued on ctx->stream is done.
void release_plan(dt_ctx *ctx, std::shared_ptr<void> &plan);

// Frees the device memory of every sparse tensor still attached to ctx and
// detaches it (called by dt_ctx_destroy).
void detach_sptensors(dt_ctx *ctx);

// Stream-ordered device allocation owned by one call.
class DevMem {
   public:
    DevMem() = default;
    DevMem(dt_ctx *ctx, size_t bytes) { alloc(ctx, bytes); }
    DevMem(const DevMem &) = delete;
    DevMem &operator=(const DevMem &) = delete;
    DevMem(DevMem &&o) noexcept { swap(o); }
    DevMem &operator=(DevMem &&o) noexcept {
        release();
        swap(o);
        return *this;
    }
    ~DevMem() { release(); }
    void alloc(dt_ctx *ctx, size_t bytes);
    void release();
    template <class T>
    T *as() const { return static_cast<T *>(p_); }
    void *get() const { return p_; }
    size_t bytes() const { return bytes_; }

   private:
    void swap(DevMem &o) {
        std::swap(p_, o.p_);
        std::swap(bytes_, o.bytes_);
        std::swap(ctx_, o.ctx_);
    }
    void *p_ = nullptr;
    size_t bytes_ = 0;
    dt_ctx *ctx_ = nullptr;
};

// A host buffer copied to a new device buffer in ctx->kCopyChunks chunks on
// the context's copy stream (created on first use), all issued by start();
// wait(c) makes the context stream wait for chunk c.  Chunks are multiples of
// 1024 elements of `esz` bytes.
struct ChunkedUpload {
    DevMem dst;
    int64_t n = 0, step = 0;
    int chunks = 0;
    void start(dt_ctx *ctx, const void *host, int64_t n, size_t esz);
    void wait(dt_ctx *ctx, int c) const;
    int64_t offset(int c) const { return (int64_t)c * step; }
    int64_t length(int c) const { return std::min(step, n - offset(c)); }
};

// Queues a copy of `bytes` from device memory to a caller buffer, host or
// device (the direction from unified addressing), on ctx->stream; the caller
// synchronises once after its last copy.
void copy_out(dt_ctx *ctx, void *user, const void *src, size_t bytes);

// Queues n block copies on ctx->stream: one kernel launch when every
// destination is device memory and every address and size is a multiple of
// 8 bytes, else one copy_out per block.  Null destinations are skipped; at
// most kMaxCopyBlocks blocks.
constexpr int kMaxCopyBlocks = 17;
void copy_blocks(dt_ctx *ctx, int n, void *const *dst, const void *const *src,
                 const size_t *bytes);

// The context's pinned read-back block (dt_ctx::kHostStageBytes bytes).
void *host_stage(dt_ctx *ctx);

// A caller buffer seen from the device: device pointers pass through, host
// pointers are staged (copied in for inputs, copied back by finish() for
// outputs).
class DevView {
   public:
    DevView(dt_ctx *ctx, const void *p, size_t bytes, bool is_input, bool is_output);
    void *ptr() const { return dptr_; }
    template <class T>
    T *as() const { return static_cast<T *>(dptr_); }
    // For host outputs: copy back and synchronise.
    void finish();

   private:
    dt_ctx *ctx_;
    void *user_;
    void *dptr_;
    size_t bytes_;
    bool output_;
    bool staged_;
    DevMem mem_;
};

// CUDA-event pairs around selected launches (opts.profile), summed at the end.
class LaunchTimer {
   public:
    explicit LaunchTimer(dt_ctx *ctx, bool on) : ctx_(ctx), on_(on) {}
    ~LaunchTimer() {
        for (auto &p : ev_) {
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
    }
    void begin() {
        if (!on_) return;
        cudaEvent_t a, b;
        DT_CUDA(cudaEventCreate(&a));
        DT_CUDA(cudaEventCreate(&b));
        ev_.push_back({a, b});
        DT_CUDA(cudaEventRecord(a, ctx_->stream));
    }
    void end(double bytes) {
        if (!on_) return;
        DT_CUDA(cudaEventRecord(ev_.back().second, ctx_->stream));
        bytes_ += bytes;
    }
    // Call after the stream has been synchronised.
    double total_ms() const {
        double t = 0.0;
        for (auto &p : ev_) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.first, p.second);
            t += ms;
        }
        return t;
    }
    int count() const { return (int)ev_.size(); }
    double bytes() const { return bytes_; }

   private:
    dt_ctx *ctx_;
    bool on_;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_;
    double bytes_ = 0.0;
};

inline int64_t prod(const int64_t *s, int n) {
    int64_t p = 1;
    for (int i = 0; i < n; i++) p *= s[i];
    return p;
}

inline unsigned ceil_div(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace dt
