// Dense HOOI drivers (FP64 and the tensor-core mixed-precision variant).
#pragma once

#include <algorithm>
#include <vector>

#include "dt_core.cuh"

namespace dt {

// The FP64 HOOI: CUDA-core TTM chain over a dimension tree, FP64 Gram and
// subspace iteration.  X may be FP64 or FP32 (read as FP32, computed in FP64).
// The GNU C library's rand() sequence after srand(seed), restated (dt_hooi.cu).
class LibcRand {
   public:
    explicit LibcRand(unsigned seed);
    int32_t next();  // in [0, 2^31 - 1], as rand()

   private:
    int32_t s_[31];
    int f_ = 3, r_ = 0;
};

struct DenseHooi {
    dt_ctx *ctx = nullptr;
    int dtype = DT_F64;
    int N = 0;
    int64_t I[16] = {}, R[16] = {};
    int64_t xsize = 0;
    dt_hooi_opts opts{};
    const void *Xdev = nullptr;
    DevMem X64;               // FP64 copy when needed
    std::vector<DevMem> U;    // I_n x R_n col-major
    DevMem S, work, flag, scal, G;
    bool allocated = false;
    // Orthonormal initial factors of the last explicit seed (DT_INIT_RANDN_LIBC).
    DevMem init_cache;
    bool init_cached = false;
    unsigned init_seed = 0;
    int hosvd_iters = 30;
    LaunchTimer *xtimer = nullptr;  // times the TTM launches that read X

    // Allocates the buffers on the first call; a later call on the same
    // object (same shapes and ranks) keeps them, so a captured sweep graph
    // stays valid.
    void setup(dt_ctx *c, const void *X, int dtype, int n, const int64_t *shape,
               const int64_t *ranks, const dt_hooi_opts &o);
    // Writes the initial factors into dst[m] (I_m x R_m col-major device
    // buffers; null: this object's U).
    void init_factors(double *const *U_user, double *const *dst = nullptr);
    // graph: replays the sweep from a captured CUDA graph (null: launch
    // directly; never used with opts.profile).
    void run(double *G_user, double *const *U_user, dt_hooi_report *rep,
             SweepGraph *graph = nullptr);

   private:
    DevMem contract(const void *t, int tdtype, int64_t *shape, int m);
    DevMem contract_all(const void *t, int tdtype, int64_t *shape, std::vector<int> modes);
    void node(int lo, int hi, const void *T, int tdtype, const int64_t *shape);
    void leaf(int n, const double *Y, const int64_t *shape);
    void sweep();
    double read_scalar(int k);
    void read_scalars(int k, int n, double *out);
    double x_pass_flop() const;
    double x_pass_bytes() const;
};

// BF16 / split-BF16 tensor-core HOOI (dt_hooi_tc.cu).
// upload: X (FP32) is still arriving from the host through it; its chunks
// are rounded to BF16 as they land (only where hooi_lowprec_tc_ok holds).
void hooi_dense_lowprec(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
                        const int64_t *ranks, const dt_hooi_opts &opts, double *G,
                        double *const *U, dt_hooi_report *report,
                        ChunkedUpload *upload = nullptr);
// Whether the tensor-core HOOI runs these shapes (otherwise it falls back to
// the FP64 engine).
bool hooi_lowprec_tc_ok(int ndim, const int64_t *shape, const int64_t *ranks);

}  // namespace dt
