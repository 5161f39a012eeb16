// Context lifetime, error reporting and host/device staging.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

#include "dt_core.cuh"

namespace dt {

static thread_local std::string g_last_error;

std::string fmt(const char *f, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof(buf), f, ap);
    va_end(ap);
    return std::string(buf);
}

void set_last_error(const std::string &msg) { g_last_error = msg; }
void clear_last_error() { g_last_error.clear(); }

void check_shape(int ndim, const int64_t *shape, const char *who) {
    DT_CHECK_ARG(ndim >= 1 && ndim <= 16 && shape, "%s: bad ndim %d", who, ndim);
    int64_t total = 1;
    for (int i = 0; i < ndim; i++) {
        DT_CHECK_ARG(shape[i] >= 1, "%s: shape[%d] = %lld must be >= 1", who, i,
                     (long long)shape[i]);
        DT_CHECK_ARG(shape[i] <= (int64_t(1) << 62) / total,
                     "%s: the element count overflows at shape[%d] = %lld", who, i,
                     (long long)shape[i]);
        total *= shape[i];
    }
}

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("DT_DISABLE_PDL");
        return !(e && e[0] == '1');
    }();
    return on;
}

namespace {
}  // namespace

bool graphs_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("DT_DISABLE_GRAPHS");
        return !(e && e[0] == '1');
    }();
    return on;
}

void release_plan(dt_ctx *ctx, std::shared_ptr<void> &plan) {
    if (!plan) return;
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    plan.reset();
}

void SweepGraph::reset() {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
    launches_ = 0;
}

void SweepGraph::run(dt_ctx *ctx, const std::function<void()> &fn) {
    const bool plain_stream = ctx->stream != nullptr && ctx->stream != cudaStreamLegacy &&
                              ctx->stream != cudaStreamPerThread;
    if (!exec_) {
        if (failed_ || !plain_stream || !graphs_enabled()) {
            fn();
            return;
        }
        const int64_t l0 = ctx->launches;
        auto give_up = [&](cudaGraph_t g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            ctx->launches = l0;
            failed_ = true;
        };
        DT_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
        cudaGraph_t g = nullptr;
        try {
            fn();
        } catch (const Error &e) {
            cudaStreamEndCapture(ctx->stream, &g);
            if (e.code == DT_ERR_NOMEM) {
                // Out of memory (or over the context's cap): the call fails and
                // the next one captures again.
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                ctx->launches = l0;
                throw;
            }
            give_up(g);
            fn();
            return;
        } catch (...) {
            cudaStreamEndCapture(ctx->stream, &g);
            give_up(g);
            fn();
            return;
        }
        if (cudaStreamEndCapture(ctx->stream, &g) != cudaSuccess || !g) {
            give_up(g);
            fn();
            return;
        }
        if (cudaGraphInstantiateWithFlags(&exec_, g, 0) != cudaSuccess) {
            exec_ = nullptr;
            give_up(g);
            fn();
            return;
        }
        cudaGraphDestroy(g);
        launches_ = ctx->launches - l0;
        ctx->launches = l0;
    }
    DT_CUDA(cudaGraphLaunch(exec_, ctx->stream));
    ctx->launches += launches_;
}

void raise_smem_limit(dt_ctx *ctx, const void *kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> limits;
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = limits[{kernel, ctx->device}];
    if (bytes <= cur) return;
    DT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

void DevMem::alloc(dt_ctx *ctx, size_t bytes) {
    release();
    if (bytes == 0) return;
    if (ctx->mem_limit && ctx->mem_in_use + bytes > ctx->mem_limit)
        fail(DT_ERR_NOMEM, fmt("device allocation of %zu bytes would exceed the context's "
                               "limit (%llu of %llu bytes in use)",
                               bytes, (unsigned long long)ctx->mem_in_use,
                               (unsigned long long)ctx->mem_limit));
    const cudaError_t e = cudaMallocAsync(&p_, bytes, ctx->stream);
    if (e != cudaSuccess) {
        p_ = nullptr;
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            fail(DT_ERR_NOMEM, fmt("device allocation of %zu bytes failed", bytes));
        }
        DT_CUDA(e);
    }
    ctx_ = ctx;
    bytes_ = bytes;
    ctx->mem_in_use += bytes;
    ctx->mem_peak = std::max(ctx->mem_peak, ctx->mem_in_use);
}

void DevMem::release() {
    if (p_ && ctx_) {
        cudaFreeAsync(p_, ctx_->stream);
        ctx_->mem_in_use -= bytes_;
    }
    p_ = nullptr;
    bytes_ = 0;
}

void ChunkedUpload::start(dt_ctx *c, const void *host, int64_t count, size_t esz) {
    constexpr int kc = dt_ctx::kCopyChunks;
    if (!c->copy_stream) {
        DT_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (cudaEvent_t &e : c->copy_ev)
            DT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    n = count;
    step = std::max<int64_t>(1024, ((n + kc - 1) / kc + 1023) / 1024 * 1024);
    chunks = (int)((n + step - 1) / step);
    dst.alloc(c, (size_t)n * esz);
    // The copies follow the context stream's earlier work (dst's allocation).
    DT_CUDA(cudaEventRecord(c->copy_ev[kc], c->stream));
    DT_CUDA(cudaStreamWaitEvent(c->copy_stream, c->copy_ev[kc], 0));
    for (int q = 0; q < chunks; q++) {
        DT_CUDA(cudaMemcpyAsync(static_cast<char *>(dst.get()) + offset(q) * esz,
                                static_cast<const char *>(host) + offset(q) * esz,
                                (size_t)length(q) * esz, cudaMemcpyHostToDevice, c->copy_stream));
        DT_CUDA(cudaEventRecord(c->copy_ev[q], c->copy_stream));
    }
}

void ChunkedUpload::wait(dt_ctx *c, int q) const {
    DT_CUDA(cudaStreamWaitEvent(c->stream, c->copy_ev[q], 0));
}

DevView::DevView(dt_ctx *ctx, const void *p, size_t bytes, bool is_input, bool is_output)
    : ctx_(ctx), user_(const_cast<void *>(p)), dptr_(nullptr), bytes_(bytes),
      output_(is_output), staged_(false) {
    if (bytes == 0) return;
    if (!p) fail(DT_ERR_ARG, "null buffer");
    if (is_device_ptr(p)) {
        dptr_ = user_;
        return;
    }
    staged_ = true;
    mem_.alloc(ctx, bytes);
    dptr_ = mem_.get();
    if (is_input)
        DT_CUDA(cudaMemcpyAsync(dptr_, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
}

void copy_out(dt_ctx *ctx, void *user, const void *src, size_t bytes) {
    if (bytes == 0) return;
    if (!user) fail(DT_ERR_ARG, "null output buffer");
    DT_CUDA(cudaMemcpyAsync(user, src, bytes, cudaMemcpyDefault, ctx->stream));
}

namespace {

struct BlockList {
    const unsigned long long *src[kMaxCopyBlocks];
    unsigned long long *dst[kMaxCopyBlocks];
    long long words[kMaxCopyBlocks];
    int count;
};

// Every block in one grid-stride pass: 8-byte words, consecutive threads on
// consecutive words.
__global__ void copy_blocks_kernel(BlockList b) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < b.count; k++)
        for (long long i = t; i < b.words[k]; i += stride) b.dst[k][i] = b.src[k][i];
}

// Device (or managed) memory of the context's own GPU: a kernel there may
// store to it without peer access.
bool is_local_device_ptr(const dt_ctx *ctx, const void *p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) &&
           attr.device == ctx->device;
}

}  // namespace

void copy_blocks(dt_ctx *ctx, int n, void *const *dst, const void *const *src,
                 const size_t *bytes) {
    DT_CHECK_ARG(n >= 0 && n <= kMaxCopyBlocks, "copy_blocks: %d blocks", n);
    BlockList b{};
    bool one_launch = true;
    long long most = 0;
    for (int k = 0; k < n; k++) {
        if (!dst[k] || bytes[k] == 0) continue;
        const bool aligned = (reinterpret_cast<uintptr_t>(dst[k]) | reinterpret_cast<uintptr_t>(src[k]) |
                              bytes[k]) % 8 == 0;
        if (!aligned || !is_local_device_ptr(ctx, dst[k])) {
            one_launch = false;
            break;
        }
        b.src[b.count] = static_cast<const unsigned long long *>(src[k]);
        b.dst[b.count] = static_cast<unsigned long long *>(dst[k]);
        b.words[b.count] = (long long)(bytes[k] / 8);
        most = std::max(most, b.words[b.count]);
        b.count++;
    }
    if (!one_launch) {
        for (int k = 0; k < n; k++)
            if (dst[k]) copy_out(ctx, dst[k], src[k], bytes[k]);
        return;
    }
    if (b.count == 0) return;
    const int threads = 256;
    const long long want = (most + threads - 1) / threads;
    const unsigned blocks = (unsigned)std::max(1LL, std::min<long long>(want, 2LL * ctx->num_sms));
    DT_LAUNCH(ctx, copy_blocks_kernel, blocks, threads, 0, b);
}

void *host_stage(dt_ctx *ctx) {
    if (!ctx->host_stage)
        DT_CUDA(cudaHostAlloc(&ctx->host_stage, dt_ctx::kHostStageBytes, cudaHostAllocDefault));
    return ctx->host_stage;
}

void DevView::finish() {
    if (output_ && staged_ && bytes_) {
        DT_CUDA(cudaMemcpyAsync(user_, dptr_, bytes_, cudaMemcpyDeviceToHost, ctx_->stream));
        DT_CUDA(cudaStreamSynchronize(ctx_->stream));
    }
}

}  // namespace dt

using namespace dt;

extern "C" {

const char *dt_last_error(void) { return g_last_error.c_str(); }

int dt_ctx_create(int device, dt_ctx **out) {
    return guard([&] {
        DT_CHECK_ARG(out, "dt_ctx_create: null output pointer");
        int n = 0;
        DT_CUDA(cudaGetDeviceCount(&n));
        DT_CHECK_ARG(device >= 0 && device < n, "dt_ctx_create: device %d out of range (%d)",
                     device, n);
        DT_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        DT_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10)
            fail(DT_ERR_UNSUPPORTED,
                 fmt("device %d is sm_%d%d; this library is built for sm_100a", device,
                     prop.major, prop.minor));
        auto *ctx = new dt_ctx();
        ctx->device = device;
        ctx->num_sms = prop.multiProcessorCount;
        // Keep freed stream-ordered allocations cached in the device's pool:
        // with the default threshold of 0 every synchronisation returns them
        // to the driver and the next cudaMallocAsync has to map pages again.
        cudaMemPool_t pool;
        DT_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = ~0ULL;
        DT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        DT_CUDA(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
        ctx->stream = ctx->own_stream;
        DT_CUDA(cudaEventCreate(&ctx->ev_start));
        DT_CUDA(cudaEventCreate(&ctx->ev_stop));
        *out = ctx;
    });
}

int dt_ctx_destroy(dt_ctx *ctx) {
    return guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->device);
        detach_sptensors(ctx);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        ctx->hooi_plan_fp64.reset();
        ctx->hooi_plan_mixed.reset();
        ctx->batched.reset();
        ctx->summary.reset();
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
        if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
        if (ctx->copy_stream) {
            cudaStreamSynchronize(ctx->copy_stream);
            for (cudaEvent_t e : ctx->copy_ev)
                if (e) cudaEventDestroy(e);
            cudaStreamDestroy(ctx->copy_stream);
        }
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        if (ctx->host_stage) cudaFreeHost(ctx->host_stage);
        delete ctx;
    });
}

int dt_ctx_set_stream(dt_ctx *ctx, void *stream) {
    return guard([&] {
        check_ctx(ctx);
        ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    });
}

int dt_ctx_set_mem_limit(dt_ctx *ctx, uint64_t bytes) {
    return guard([&] {
        check_ctx(ctx);
        ctx->mem_limit = bytes;
    });
}

int dt_ctx_mem_usage(dt_ctx *ctx, uint64_t *in_use, uint64_t *peak) {
    return guard([&] {
        check_ctx(ctx);
        if (in_use) *in_use = ctx->mem_in_use;
        if (peak) *peak = ctx->mem_peak;
    });
}

int dt_ctx_synchronize(dt_ctx *ctx) {
    return guard([&] {
        check_ctx(ctx);
        DT_CUDA(cudaSetDevice(ctx->device));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int64_t dt_ctx_kernel_launches(dt_ctx *ctx) { return ctx ? ctx->launches : -1; }

}  // extern "C"
