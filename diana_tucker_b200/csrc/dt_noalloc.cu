// dt_gram_f64_noalloc: the FP64 Gram G = X_(mode) X_(mode)^T of dt_gram_f64,
// computed without allocating any memory.  The split-K partial tiles that
// dt_gram_f64 keeps in a stream-ordered allocation live here in a fixed,
// library-owned device array instead.
//
// Who needs it: callers that cannot call cudaMalloc / cudaMallocAsync while
// they run -- a host framework that owns and budgets the whole device heap
// (its own caching allocator or a fixed arena) and forbids side allocations,
// code on a latency-critical path where an allocation may synchronise the
// device or fail under fragmentation, and callers with no allocator to link.
// They pass device buffers for the input and the output; the scratch is
// `g_noalloc_scratch` below.
//
// What a caller has to know:
//  * the array is a file-scope `static __device__` object: every GPU that
//    loads this library holds it (16 MiB) until the process exits;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress, with that device current, and caches it per device
//    and CUDA context; make that first call before any stream capture.  A
//    device reset (cudaDeviceReset) gives the device a new context, and the
//    next call looks the array up again, so it never uses a stale address;
//  * every call on a device shares the one array, which keeps the last call's
//    contents.  Each call overwrites every partial tile it reads, so nothing
//    has to start at zero; two calls whose kernels overlap on the GPU (two
//    streams, two host threads) race on the array -- serialise them;
//  * X and G must be device memory of the context's GPU (staging host buffers
//    would allocate); the mode size is at most 1024, so that the partial Grams
//    the split-K schedule needs fit the array.
#include <map>
#include <mutex>

#include "dt_kernels.cuh"

namespace dt {
namespace {

constexpr int64_t kScratchDoubles = int64_t(1) << 21;  // 16 MiB
constexpr int64_t kMaxModeSize = 1024;                 // 2 * 1024^2 doubles = 16 MiB
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

using CtxGetCurrentFn = int (*)(void **);

// The driver's current context (cuCtxGetCurrent, fetched from the driver at
// run time like the rest of the library's driver calls).
void *current_context() {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        DT_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess)
            fail(DT_ERR_CUDA, "cuCtxGetCurrent is not available from the driver");
        fn = reinterpret_cast<CtxGetCurrentFn>(p);
    }
    void *c = nullptr;
    if (fn(&c) != 0) fail(DT_ERR_CUDA, "cuCtxGetCurrent failed");
    return c;
}

// Device address of the scratch array on `device`, which must be current.
// On the host `g_noalloc_scratch` is only a stand-in for the device object
// and is never passed to a kernel.  Cached per (device, context): a reset
// device has a new context, where the module and its array are loaded anew.
double *scratch_address(int device) {
    static std::mutex mu;
    static std::map<std::pair<int, void *>, double *> cache;
    std::lock_guard<std::mutex> lock(mu);
    const std::pair<int, void *> key(device, current_context());
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    double *p = nullptr;
    DT_CUDA(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch));
    DT_CHECK_ARG(p != nullptr, "dt_gram_f64_noalloc: cudaGetSymbolAddress gave a null address");
    cache[key] = p;
    return p;
}

}  // namespace
}  // namespace dt

using namespace dt;

extern "C" {

int dt_gram_f64_noalloc(dt_ctx *ctx, const double *X, int ndim, const int64_t *shape, int mode,
                        double *G) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(X && G, "dt_gram_f64_noalloc: bad arguments");
        check_shape(ndim, shape, "dt_gram_f64_noalloc");
        DT_CHECK_ARG(mode >= 0 && mode < ndim, "dt_gram_f64_noalloc: mode %d out of range", mode);
        const int64_t I = shape[mode];
        DT_CHECK_ARG(I <= kMaxModeSize,
                     "dt_gram_f64_noalloc: mode size %lld exceeds the limit of %lld (its "
                     "partial Grams must fit the fixed 16 MiB scratch)",
                     (long long)I, (long long)kMaxModeSize);
        DT_CUDA(cudaSetDevice(ctx->device));
        DT_CHECK_ARG(is_device_ptr(X) && is_device_ptr(G),
                     "dt_gram_f64_noalloc: X and G must be device memory");
        int64_t L = 1, B = 1;
        for (int m = 0; m < mode; m++) L *= shape[m];
        for (int m = mode + 1; m < ndim; m++) B *= shape[m];
        double *scratch = scratch_address(ctx->device);
        ttt_f64_scratch(ctx, X, X, L, I, I, B, G, scratch, kScratchDoubles);
    });
}

}  // extern "C"
