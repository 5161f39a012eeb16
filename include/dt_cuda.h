/*
 * dt_cuda.h -- C ABI of libdt_cuda.so, the B200 (sm_100a) implementation of
 * DIANA-Tucker's HOOI-ALS hot path.
 *
 * Conventions (mirroring the reference's Operator<double> seam,
 * include/operator.hpp:8-70, and its Tensor<Ty> layout, template/tensor_mpi.tpp:49-53):
 *  - dense tensors are column-major (mode 0 fastest), shapes are int64;
 *  - a matrix argument "J x I col-major" is stored with its row index fastest;
 *  - every pointer may be HOST or DEVICE memory of the context's GPU; host
 *    buffers are staged through the context (the reference's buffers are
 *    malloc'd host memory, operator_cpu.tpp:6-12);
 *  - every entry point returns 0 on success and a nonzero DT_ERR_* code on
 *    failure; dt_last_error() then describes the failure.  This replaces the
 *    reference's error()/assert -> exit() convention (include/logger.hpp:75-123);
 *  - a context is bound to one device and one CUDA stream; use one context
 *    per host thread.
 *  - the world has size 1: the reference's MPI distribution
 *    (DistributionCartesianBlock, communicator.tpp) collapses to one GPU.
 */
#ifndef DT_CUDA_H
#define DT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DT_API __attribute__((visibility("default")))
#else
#define DT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define DT_OK 0
#define DT_ERR_ARG 1       /* invalid argument (shape mismatch, bad mode, ...) */
#define DT_ERR_CUDA 2      /* a CUDA runtime / driver call failed */
#define DT_ERR_NOMEM 3     /* device allocation failed */
#define DT_ERR_NUMERIC 4   /* breakdown (singular matrix, non-SPD Gram, NaN) */
#define DT_ERR_UNSUPPORTED 5
#define DT_ERR_TIMEOUT 6   /* a bounded device wait ran out: the kernel recorded it
                              and returned, and the context stays usable */

/* ---- element types and options --------------------------------------- */
#define DT_F64 0
#define DT_F32 1

/* HOOI initialisation */
#define DT_INIT_RANDN_LIBC 0 /* reference: srand(seed); Util::randn() per element,
                                column-major I_n x R_n, then reduced_QR
                                (hooi_als.tpp:74-81, util.cpp:10-18) */
#define DT_INIT_HOSVD 1      /* leading R_n eigenvectors of X_(n) X_(n)^T */
#define DT_INIT_GIVEN 2      /* factors supplied by the caller in U */
#define DT_SEED_KEEP 0xFFFFFFFFu

/* HOOI arithmetic for the TTM chain and the Gram (the eigensolve / QR, the
 * fit and the final core projection are FP64 in every mode). */
#define DT_PREC_FP64 0   /* FP64 CUDA-core kernels throughout (the drop-in) */
#define DT_PREC_BF16 1   /* tcgen05 BF16 x BF16 -> FP32 TTM chain and Gram */
#define DT_PREC_BF16X2 2 /* tcgen05 with split hi+lo BF16 operands (~2^-16) */
#define DT_PREC_BF16XH 3 /* X rounded once to BF16 (2 bytes per element per pass);
                            U, the intermediates and the Grams split hi+lo */

typedef struct dt_ctx dt_ctx;

typedef struct {
    int init;           /* DT_INIT_* */
    unsigned seed;      /* for DT_INIT_RANDN_LIBC: the draws of srand(seed)
                           followed by rand() (the library's restatement of the
                           C library's generator: the process's rand() state is
                           left alone, and a context reuses the factors of a
                           seed it has drawn); DT_SEED_KEEP continues the
                           process's current rand() sequence, as the
                           reference's HOOI_ALS does after the caller's srand */
    int max_sweeps;     /* reference: max_iter */
    double tol;         /* stop when |res_k - res_{k-1}| < tol; <= 0 runs max_sweeps */
    int inner_iters;    /* subspace iterations per mode (reference ALS_: 5) */
    int precision;      /* DT_PREC_* */
    int refine_sweeps;  /* BF16 modes: the last sweeps (after the tol test first
                           passes) run with hi+lo operands; 0 = none */
    int verbose;        /* print one line per sweep to stderr */
    int profile;        /* record CUDA events around every TTM launch that
                           streams X (reported as ttm_x_*) */
} dt_hooi_opts;

#define DT_MAX_HIST 256
typedef struct {
    int sweeps;                   /* sweeps run */
    double x_norm;                /* ||X||_F (FP64) */
    double g_norm;                /* ||G||_F of the returned core (FP64 projection) */
    double residual;              /* sqrt(1 - ||G||^2/||X||^2) */
    double device_ms;             /* CUDA-event time of the whole decomposition */
    double res_hist[DT_MAX_HIST]; /* per-sweep residual as tracked by the sweep */
    int kernel_launches;          /* kernels launched by the decomposition */
    int precision_used;           /* DT_PREC_* actually run (a tensor-core request
                                     falls back to FP64 for shapes outside the
                                     TMA / UMMA layout rules) */
    int ttm_x_launches;           /* with opts.profile: TTM launches that read X */
    double ttm_x_ms;              /* ... their summed CUDA-event time */
    double ttm_x_bytes;           /* ... their summed algorithmic bytes
                                     (X read + output written + factor read) */
} dt_hooi_report;

/* ---- context ---------------------------------------------------------- */
/* No reference counterpart (the reference has no device state). */
DT_API int dt_ctx_create(int device, dt_ctx **ctx);
DT_API int dt_ctx_destroy(dt_ctx *ctx);
/* Run all work of this context on the given cudaStream_t (NULL = the
 * context's own non-blocking stream; to order work after the legacy default
 * stream, pass cudaStreamLegacy). */
DT_API int dt_ctx_set_stream(dt_ctx *ctx, void *stream);
DT_API int dt_ctx_synchronize(dt_ctx *ctx);
/* Message of the last failure on the calling thread ("" if none). */
DT_API const char *dt_last_error(void);
/* Number of this library's kernels launched by ctx since creation. */
DT_API int64_t dt_ctx_kernel_launches(dt_ctx *ctx);
/* A cap on the device memory this context's calls allocate (bytes; 0 = no
 * cap).  A call whose allocation would cross it fails with DT_ERR_NOMEM before
 * allocating, frees what it holds and leaves the context usable (the
 * reference's Operator::alloc ends the process instead, operator_cpu.tpp:6-12). */
DT_API int dt_ctx_set_mem_limit(dt_ctx *ctx, uint64_t bytes);
/* Device bytes the context holds now (cached plans included) and at most
 * since creation. */
DT_API int dt_ctx_mem_usage(dt_ctx *ctx, uint64_t *in_use, uint64_t *peak);
/* Self-test of the bounded device waits: one kernel waits on an mbarrier that
 * nothing arrives on, for limit_cycles SM clock cycles (<= the 2e9 budget of
 * every wait in the library), records the timeout and returns.  Returns
 * DT_ERR_TIMEOUT, as a real wait that ran out does; the context stays usable. */
DT_API int dt_selftest_wait_timeout(dt_ctx *ctx, int64_t limit_cycles);

/* ---- operator-level entry points -------------------------------------- */
/* Y = X x_mode M, M is J x I_mode col-major, Y has shape[mode] replaced by J.
 * Replaces Function::ttm (template/function/tensor.tpp:272-335) at world size 1,
 * without its tenmatt/mattten permute copies (operator_cpu.tpp:83-135). */
DT_API int dt_ttm_f64(dt_ctx *ctx, const double *X, int ndim, const int64_t *shape, int mode,
               const double *M, int64_t J, double *Y);

/* G = X_(mode) X_(mode)^T, I_mode x I_mode col-major.
 * Replaces Function::gram (tensor.tpp:18-120). */
DT_API int dt_gram_f64(dt_ctx *ctx, const double *X, int ndim, const int64_t *shape, int mode,
                double *G);

/* dt_gram_f64 without allocating: no counterpart in the reference.  For
 * callers that cannot call cudaMalloc while they run (a host framework that
 * owns the device heap, a latency-critical path where an allocation may
 * synchronise or fail).  X and G must be device memory of the context's GPU;
 * shape[mode] <= 1024.  The split-K partial tiles live in a fixed 16 MiB
 * `static __device__` array that every GPU loading this library holds until
 * exit.  The first call on a device looks the array up (cudaGetSymbolAddress):
 * make it before any stream capture.  The address is cached per device and
 * CUDA context, so after a device reset the next call looks it up again.
 * Calls share the array, so calls whose kernels overlap on the GPU race;
 * serialise them. */
DT_API int dt_gram_f64_noalloc(dt_ctx *ctx, const double *X, int ndim, const int64_t *shape,
                               int mode, double *G);

/* C = A_(mode) B_(mode)^T, shapeA[mode] x shapeB[mode] col-major; the other
 * modes of A and B must agree.  Replaces Function::ttt_except (tensor.tpp:132-259). */
DT_API int dt_ttt_except_f64(dt_ctx *ctx, const double *A, const int64_t *shapeA, const double *B,
                      const int64_t *shapeB, int ndim, int mode, double *C);

/* ||X||_F.  Replaces Function::fnorm (tensor.tpp:467-480) / Operator::fnorm
 * (operator_double.cpp:74-82). */
DT_API int dt_fnorm_f64(dt_ctx *ctx, const double *X, int64_t n, double *out);

/* C = op(A) op(B), column-major; trans = 0 (N) or 1 (T).  (m,n,k) as in the
 * reference: NN C(m x n) = A(m x k) B(k x n); NT C = A(m x k) B(n x k)^T;
 * TN C = A(k x m)^T B(k x n).  Replaces Operator::matmulNN/NT/TN
 * (operator_double.cpp:157-216). */
DT_API int dt_matmul_f64(dt_ctx *ctx, int transA, int transB, int64_t m, int64_t n, int64_t k,
                  const double *A, const double *B, double *C);

/* Householder QR of an m x n (m >= n) col-major matrix: Q m x n, R n x n
 * (R may be NULL).  Same reflector convention as LAPACK dgeqrf/dorgqr.
 * Replaces Operator::QR (operator_double.cpp:131-155). */
DT_API int dt_reduced_qr_f64(dt_ctx *ctx, const double *A, int64_t m, int64_t n, double *Q,
                      double *R);

/* Inverse of an n x n matrix by LU with partial pivoting.
 * Replaces Operator::inverse (operator_double.cpp:84-103); a zero pivot
 * returns DT_ERR_NUMERIC where the reference only warns. */
DT_API int dt_inverse_f64(dt_ctx *ctx, const double *A, int64_t n, double *Ainv);

/* Modified Gram-Schmidt over the len1 rows of a len1 x len2 col-major matrix,
 * in place.  Replaces Operator::orth2 (operator_double.cpp:248-277). */
DT_API int dt_orth2_f64(dt_ctx *ctx, double *A, int64_t len1, int64_t len2);

/* ALS_ leading-subspace step for mode n of the TTM-chain output Y, from the
 * I_n x R col-major L0: Q = orth((Y_(n) Y_(n)^T)^iters L0).  Replaces
 * Algorithm::Tucker::ALS_ (hooi_als.tpp:7-34), whose 5 steps span the same
 * subspace. */
DT_API int dt_als_f64(dt_ctx *ctx, const double *Y, int ndim, const int64_t *shape, int mode,
               const double *L0, int64_t R, int iters, double *Q);

/* ---- tensor-core (sm_100a tcgen05) operators ---------------------------- */
/* Y = X x_mode U^T on the tensor cores: X (FP32, column-major) is rounded to
 * BF16 (split = 0) or split into BF16 hi + lo (split = 1), U (shape[mode] x J
 * col-major, FP64) likewise; FP32 accumulation; Y (FP32) folded like X with
 * shape[mode] -> J.  The mixed-precision form of Function::ttm
 * (tensor.tpp:272-335) used by the BF16 HOOI.  DT_ERR_UNSUPPORTED when the
 * layout falls outside the TMA rules (mode 0 needs shape[0] % 8 == 0; other
 * modes need prod_{m<mode} shape[m] >= 64 and % 8 == 0; J <= 32). */
DT_API int dt_ttm_tc(dt_ctx *ctx, const float *X, int ndim, const int64_t *shape, int mode,
                     const double *U, int64_t J, int split, float *Y);

/* S (I x I, FP64) = Y Y^T for a row-major I x K FP32 Y, on the tensor cores
 * (BF16 or split hi+lo operands, FP32 accumulation, FP64 reduction of the
 * split-K partials).  The Gram of Function::gram (tensor.tpp:18-120) for
 * I <= 128, K % 8 == 0. */
DT_API int dt_gram_tc(dt_ctx *ctx, const float *Y, int64_t I, int64_t K, int split, double *S);

/* ---- learned warm start (no counterpart in the reference, which starts
 * HOOI from random factors, hooi_als.tpp:74-81) -------------------------
 * A linear autoencoder over factor columns of length n: encoder E (k x n),
 * decoder D (n x k), both col-major FP64, k <= 32. */

/* Loss |D E U - U|^2 / N over the N columns of U (n x N col-major) and its
 * gradients dE (k x n), dD (n x k): one forward and backward pass. */
DT_API int dt_ws_loss_grad(dt_ctx *ctx, const double *U, int64_t n, int64_t N, int k,
                           const double *E, const double *D, double *loss, double *gE,
                           double *gD);

/* Trains E and D from seeded Gaussian weights with `steps` full-batch Adam
 * steps (rate lr) on the columns of U; loss_hist (steps values, may be NULL)
 * receives the loss before each step. */
DT_API int dt_ws_train(dt_ctx *ctx, const double *U, int64_t n, int64_t N, int k, int steps,
                       double lr, uint64_t seed, double *E, double *D, double *loss_hist);

/* Initial factors for dense HOOI from the decoder D (n x k): sketch
 * X x_m orth(D)^T over every mode (k^ndim values, one pass over X), leading
 * R_m subspaces of the sketch refined by up to sketch_sweeps HOOI sweeps on
 * the sketch, decoded to U[m] (n x R_m col-major).  Every mode has size n;
 * R_m <= k.  fit_sketch = |sketch|^2 / |X|^2, fit_init = |X x_m U_m^T|^2 / |X|^2. */
DT_API int dt_ws_init(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
                      const int64_t *ranks, const double *D, int k, int sketch_sweeps,
                      double *const *U, double *fit_sketch, double *fit_init);

/* ---- dense HOOI ------------------------------------------------------- */
/* Tucker decomposition of X (dtype DT_F64 or DT_F32, column-major) with the
 * given ranks.  G (prod ranks, col-major) and U[n] (shape[n] x ranks[n]
 * col-major) receive the result; with DT_INIT_GIVEN, U holds the initial
 * factors on entry.  Either may be NULL.  Replaces
 * Algorithm::Tucker::HOOI_ALS (hooi_als.tpp:64-123). */
DT_API int dt_hooi_dense(dt_ctx *ctx, const void *X, int dtype, int ndim, const int64_t *shape,
                  const int64_t *ranks, const dt_hooi_opts *opts, double *G,
                  double *const *U, dt_hooi_report *report);

/* Fills opts with the reference's behaviour: random libc init, 5 inner
 * iterations, FP64, no tolerance. */
DT_API void dt_hooi_default_opts(dt_hooi_opts *opts);
/* The first n values rand() returns after srand(seed) in the GNU C library, as
 * the library's own restatement of that generator computes them: the draws of
 * DT_INIT_RANDN_LIBC with an explicit seed, which leave the process's rand()
 * state untouched.  No device needed; for checking against the C library. */
DT_API int dt_libc_rand_sequence(unsigned seed, int64_t n, int32_t *out);

/* ---- batched dense HOOI ------------------------------------------------ */
typedef struct {
    double device_ms;     /* CUDA-event time of the graph launch */
    int block_threads;    /* threads per CTA (autotuned when 0 was requested) */
    int grid;             /* persistent CTAs (resident CTAs per SM x SMs) */
    int kernel_launches;
    int pack;             /* 0: one tensor per CTA; 1: tensors with largest mode
                             <= 37 two to a CTA; 2: also those <= 21 four to a CTA */
    int items;            /* work items (CTA-sized units) of the launch */
    int candidates_timed; /* configurations the autotuner timed (0: cached) */
    double tune_best_ms;  /* the autotuner's fastest and slowest sample times */
    double tune_worst_ms;
    int graph_reused;     /* 1: an instantiated graph of an earlier call replayed */
} dt_batched_report;

/* HOOI of `count` independent 3-way tensors in one persistent launch (CUDA
 * graph: queue reset + kernel).  Tensor t has shape shapes[3t..3t+2] (each
 * <= 64), ranks ranks[3t..3t+2] (each <= 8 and <= the mode size), FP32 data
 * at X + x_offsets[t] (column-major), initial factors (I_n x R_n col-major,
 * FP64) at U + u_offsets[3t+n], overwritten with the result; the core goes to
 * G + g_offsets[t] and the relative error sqrt(1 - ||G||^2/||X||^2) to
 * relerr[t].  `sweeps` HOOI sweeps with `inner_iters` ALS_ steps per mode, in
 * FP64.  Tensors are ordered longest first and small ones may share a CTA.
 * block_threads = 0 autotunes the block size and the packing on a sample of
 * the batch (cached per batch signature); 128/256/512 fix the block size and
 * pack the small tensors two and four to a CTA.  The instantiated graph is kept on the context and
 * replayed by later calls with the same launch shape.  Batched form of
 * Algorithm::Tucker::HOOI_ALS (hooi_als.tpp:64-123); no reference counterpart
 * for the batching. */
DT_API int dt_hooi_batched(dt_ctx *ctx, int count, const int64_t *shapes, const int64_t *ranks,
                           const float *X, const int64_t *x_offsets, int sweeps, int inner_iters,
                           double *U, const int64_t *u_offsets, double *G,
                           const int64_t *g_offsets, double *relerr, int block_threads,
                           dt_batched_report *report);

/* ---- sparse tensors --------------------------------------------------- */
typedef struct dt_sptensor dt_sptensor;

/* Uploads a COO tensor (idx[m][e], 0-based int64; vals[e] FP64) and builds,
 * on the device, one copy of the nonzeros sorted by each mode with its row
 * pointer (the per-mode CSR that SpTensor::index_buffer declares,
 * include/sp_tensor.hpp:16-24, and ttmc_mTL reads as v_index_buffer).
 * Replaces SpTensor<Ty>::SpTensor(data_buffer<Ty>*) (sp_tensor.hpp:71-240)
 * at world size 1. */
DT_API int dt_sptensor_create(dt_ctx *ctx, int64_t nnz, int ndim, const int64_t *const *idx,
                       const double *vals, const int64_t *shape, dt_sptensor **sp);
DT_API int dt_sptensor_destroy(dt_sptensor *sp);
/* ||A||_F of the nonzeros.  Replaces Function::fnorm(SpTensor) (sp_tensor.tpp:6-14). */
DT_API int dt_sp_fnorm(dt_ctx *ctx, const dt_sptensor *sp, double *out);

/* Factors are TRANSPOSED as in the reference (sp_hooi_als.tpp:80): Ut[m] is
 * R_m x I_m col-major, i.e. factor row i is contiguous at Ut[m] + i*R_m.
 * P = prod_{m != mode} R_m, Kronecker index with the lowest mode fastest
 * (sp_tensor.tpp:367-417). */

/* L (P x R_mode col-major) = Y_(mode)^T U_mode.  Replaces Function::ttmc_mTR
 * (sp_tensor.tpp:236-286), intended semantics. */
DT_API int dt_sp_ttmc_mTR(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                   const int64_t *R, int mode, double *L);
/* out (R_mode x I_mode col-major) = (Y_(mode) L)^T.  Replaces
 * Function::ttmc_mTL (sp_tensor.tpp:288-365). */
DT_API int dt_sp_ttmc_mTL(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                   const int64_t *R, int mode, const double *L, double *out);
/* Y_(mode) rows: Y is I_mode x P row-major (row i contiguous).  The TTMc
 * itself (add_outer_product_all over each row, sp_tensor.tpp:367-417). */
DT_API int dt_sp_ttmc_rows(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                    const int64_t *R, int mode, double *Y);

/* Y = A x_{m in idx} M_m as a dense column-major tensor: mode m has extent
 * J[m] when m is listed in idx (nidx distinct modes, any order) and I_m
 * otherwise.  M[m] is J[m] x I_m col-major (host or device; entries of
 * modes outside idx are not read and may be NULL).  Duplicate coordinates add
 * up; no floating-point atomics (rows of the kept modes are summed in a fixed
 * order).  Replaces Function::ttmc(SpTensor, M, idx, distribution, to_permu)
 * (sp_tensor.tpp:16-192, add_outer_product :419-450) at world size 1; the
 * reference's to_permu only picks its internal buffer order, so it has no
 * counterpart.  The grouping of the nonzeros by their kept coordinates is
 * built on the first call per set of kept modes and kept on the tensor. */
DT_API int dt_sp_ttmc_dense_f64(dt_ctx *ctx, const dt_sptensor *sp, const double *const *M,
                                const int64_t *J, const int *idx, int nidx, double *Y);
/* The same result by Function::mettmc (sp_tensor.tpp:194-211): the modes of
 * idx sorted by I_m / J_m (integer quotient, ascending; ties keep the given
 * order), the sparse TTMc of all but the first `level` of them, then
 * Function::ttm (dt_ttm_f64's kernels) of those `level` modes in that order.
 * 0 <= level <= nidx. */
DT_API int dt_sp_mettmc_f64(dt_ctx *ctx, const dt_sptensor *sp, const double *const *M,
                            const int64_t *J, const int *idx, int nidx, int level, double *Y);

/* Sparse HOOI power sweeps: per mode L = Y_(n)^T U_n, U_n <- orth(Y_(n) L);
 * core G (P_{N-1} x R_{N-1} col-major = the core tensor col-major) after the
 * sweeps.  Ut holds the initial transposed factors on entry and the final
 * ones on exit.  The report's ttm_x_* fields time the TTMc launches (CUDA
 * events) with their algorithmic bytes.  Replaces
 * Algorithm::SpTucker::Sp_HOOI_ALS (sp_hooi_als.tpp:67-118). */
DT_API int dt_sp_hooi(dt_ctx *ctx, const dt_sptensor *sp, const int64_t *R, int max_sweeps,
               double *const *Ut, double *G, dt_hooi_report *report);

/* ---- Summary profiler ---------------------------------------------------- */
/* The reference's Summary (include/summary.hpp:27-60, src/summary.cpp):
 * enabling starts "{Main}" (Summary::init); library operations then record
 * named, nested ranges as CUDA events on the context's stream, each with its
 * flop and byte counts, which also count towards the enclosing range
 * (Summary::start / Summary::end).  Off by default. */
DT_API int dt_summary_enable(dt_ctx *ctx, int on);
/* Drops the recorded ranges. */
DT_API int dt_summary_reset(dt_ctx *ctx);
/* Closes the open ranges and writes the table of Summary::print_summary
 * (src/summary.cpp:100-206: per name Time(s), Time C.(%), Number,
 * Avg. Time(s), GFlop/s, Bandw.(GB/s)) into buf, NUL-terminated and cut to
 * size bytes; *needed is the full length + 1.  Recording then restarts. */
DT_API int dt_summary_table(dt_ctx *ctx, char *buf, int64_t size, int64_t *needed);

/* ---- .tns ingest -------------------------------------------------------- */
typedef struct dt_tns dt_tns;

/* Reads a .tns text file ("i_1 ... i_N value" per line, 1-based indices,
 * separated by spaces or tabs) and parses it on the device: a newline scan,
 * one thread per line, dims = max index + 1 per mode, blank lines skipped.
 * Replaces read_data<double> (src/read_data.cpp:36-129) at world size 1, which
 * parses on one host thread.  The reference's read_double takes digits and
 * '.' only (read_data.cpp:24-33); values here may also carry a sign and an
 * exponent.  A line with another token count, an index below 1 or a token
 * that is not a number fails with DT_ERR_ARG naming the line. */
DT_API int dt_tns_read(dt_ctx *ctx, const char *path, dt_tns **out, int *ndim, int64_t *nnz);
/* The same on a .tns image already in memory (host or device bytes). */
DT_API int dt_tns_parse(dt_ctx *ctx, const char *bytes, int64_t size, dt_tns **out, int *ndim,
                        int64_t *nnz);
/* dims[ndim]; idx[m] (nnz 0-based int64 each) and vals (nnz FP64), host or
 * device, in file order.  Any argument may be NULL to skip it.  The
 * data_buffer<double> fields (include/read_data.hpp:9-17). */
DT_API int dt_tns_copy(dt_ctx *ctx, const dt_tns *t, int64_t *dims, int64_t *const *idx,
                       double *vals);
/* The sparse tensor of the parsed nonzeros, built from the device copy
 * (SpTensor<Ty>::SpTensor(data_buffer<Ty>*), sp_tensor.hpp:71-240). */
DT_API int dt_tns_to_sptensor(dt_ctx *ctx, const dt_tns *t, dt_sptensor **sp);
DT_API int dt_tns_destroy(dt_tns *t);

#ifdef __cplusplus
}
#endif
#endif /* DT_CUDA_H */
