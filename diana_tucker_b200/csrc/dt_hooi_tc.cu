// Mixed-precision dense HOOI on the tcgen05 tensor cores.
#include "dt_hooi.cuh"
#include "dt_kernels.cuh"

namespace dt {

void hooi_dense_lowprec(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
                        const int64_t *ranks, const dt_hooi_opts &opts, double *G,
                        double *const *U, dt_hooi_report *report) {
    (void)ctx; (void)X; (void)dtype; (void)ndim; (void)shape; (void)ranks; (void)opts;
    (void)G; (void)U; (void)report;
    fail(DT_ERR_UNSUPPORTED, "tensor-core HOOI not built yet");
}

}  // namespace dt
