// FP64 dense kernels on the CUDA cores: the stride-aware TTM, the unfolding
// GEMM behind Gram / ttt_except / matmul, and deterministic norms.
//
// The reference's Function::ttm (template/function/tensor.tpp:272-335) first
// permutes A into A_(n)^T with Operator::tenmatt (operator_cpu.tpp:83-103),
// runs dgemm, then folds back with mattten (operator_cpu.tpp:115-135).  Here the
// mode-n unfolding is never materialised: X is read as the 3-way array
// X[l, i, b] (l < prod_{m<n} I_m unit-stride, i = mode-n index with stride L,
// b the trailing modes) and the result is written straight into the folded
// layout Y[l, j, b].
#include "dt_kernels.cuh"

namespace dt {

// ---------------------------------------------------------------------------
// TTM: Y[l, j, b] = sum_i M(j, i) X[l, i, b], M(j, i) = M[j*msj + i*msi].  One CTA owns 256 "rows"
// p = l + L*b of the output and a JT-wide slice of j; X tiles (16 i x 256 p)
// are staged through shared memory so every global load is coalesced: along
// l when L > 1, along i when L == 1 (mode 0, where the contracted index is the
// contiguous one).  Each thread accumulates 2 rows x JT outputs in registers.
// ---------------------------------------------------------------------------
namespace {

constexpr int TTM_BP = 256;
constexpr int TTM_BK = 16;
constexpr int TTM_NT = 128;

template <class TX, int JT>
__global__ void __launch_bounds__(TTM_NT) ttm_kernel(const TX *__restrict__ X, int64_t L,
                                                     int64_t I, int64_t P,
                                                     const double *__restrict__ M, int64_t msj,
                                                     int64_t msi, int64_t J,
                                                     double *__restrict__ Y, int64_t kchunk,
                                                     int64_t ysize) {
    __shared__ __align__(16) double Xs[TTM_BK][TTM_BP];
    __shared__ __align__(16) double Ms[TTM_BK][JT];
    const int t = threadIdx.x;
    pdl_wait();
    const int64_t p0 = (int64_t)blockIdx.x * TTM_BP;
    const int64_t j0 = (int64_t)blockIdx.y * JT;
    const int64_t LI = L * I;
    // Split-K: blockIdx.z owns i in [ibeg, iend) and writes its own partial Y.
    const int64_t ibeg = (int64_t)blockIdx.z * kchunk;
    const int64_t iend = min(I, ibeg + kchunk);
    Y += (int64_t)blockIdx.z * ysize;

    // Loader bookkeeping for L > 1: this thread loads rows t and t + 128.
    int64_t lbase[2];
    bool lok[2];
    if (L > 1) {
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int64_t p = p0 + t + s * TTM_NT;
            lok[s] = p < P;
            const int64_t b = p / L, l = p - b * L;
            lbase[s] = l + LI * b;
        }
    }

    double acc[2][JT];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int j = 0; j < JT; j++) acc[r][j] = 0.0;

    for (int64_t i0 = ibeg; i0 < iend; i0 += TTM_BK) {
        if (L > 1) {
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int pp = t + s * TTM_NT;
#pragma unroll 4
                for (int k = 0; k < TTM_BK; k++) {
                    const int64_t i = i0 + k;
                    Xs[k][pp] = (lok[s] && i < iend) ? (double)X[lbase[s] + L * i] : 0.0;
                }
            }
        } else {
            const int k = t & (TTM_BK - 1);
            const int g = t >> 4;  // 0..7
            const int64_t i = i0 + k;
#pragma unroll 4
            for (int s = 0; s < TTM_BP / 8; s++) {
                const int pp = g + 8 * s;
                const int64_t p = p0 + pp;
                Xs[k][pp] = (p < P && i < iend) ? (double)X[p * I + i] : 0.0;
            }
        }
        for (int e = t; e < TTM_BK * JT; e += TTM_NT) {
            const int k = e / JT, j = e - (e / JT) * JT;
            const int64_t i = i0 + k, jj = j0 + j;
            Ms[k][j] = (i < iend && jj < J) ? M[jj * msj + i * msi] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < TTM_BK; k++) {
            const double2 x = *reinterpret_cast<const double2 *>(&Xs[k][2 * t]);
#pragma unroll
            for (int j = 0; j < JT; j += 2) {
                const double2 m = *reinterpret_cast<const double2 *>(&Ms[k][j]);
                acc[0][j] = fma(x.x, m.x, acc[0][j]);
                acc[0][j + 1] = fma(x.x, m.y, acc[0][j + 1]);
                acc[1][j] = fma(x.y, m.x, acc[1][j]);
                acc[1][j + 1] = fma(x.y, m.y, acc[1][j + 1]);
            }
        }
        __syncthreads();
    }

    pdl_trigger();  // dependents may launch while the outputs are stored
    const int64_t LJ = L * J;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int64_t p = p0 + 2 * t + r;
        if (p >= P) continue;
        const int64_t b = p / L, l = p - b * L;
        double *y = Y + l + LJ * b;
#pragma unroll
        for (int j = 0; j < JT; j++)
            if (j0 + j < J) y[L * (j0 + j)] = acc[r][j];
    }
}

// ---------------------------------------------------------------------------
// Pipelined TTM for the two layouts the HOOI dimension tree produces from X:
//   ROWS (L % 256 == 0): the 256 output rows of a CTA are one contiguous run
//        of l, so every k of a tile is a 16-byte-aligned contiguous segment;
//   KFAST (L == 1): the contracted index is contiguous, each row of the tile
//        is 16 consecutive i.
// Tiles move with cp.async (16 B, zero-filled past I) into a two-stage ring so
// the next K-chunk streams while this one is multiplied.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <class TX, int JT, bool KFAST>
__global__ void __launch_bounds__(TTM_NT) ttm_pipe_kernel(const TX *__restrict__ X, int64_t L,
                                                          int64_t I, int64_t P,
                                                          const double *__restrict__ M,
                                                          int64_t msj, int64_t msi, int64_t J,
                                                          double *__restrict__ Y, int64_t kchunk,
                                                          int64_t ysize) {
    constexpr int EV = 16 / sizeof(TX);              // elements per 16-byte copy
    constexpr int KROW = 16 + (KFAST ? EV : 0);      // KFAST row stride (elements), padded
    constexpr int XS_ELEMS = KFAST ? TTM_BP * KROW : TTM_BK * TTM_BP;
    extern __shared__ __align__(16) uint8_t pipe_smem[];
    auto Ms = reinterpret_cast<double(*)[TTM_BK][JT]>(pipe_smem);
    auto Xs = reinterpret_cast<TX(*)[XS_ELEMS]>(pipe_smem + 2 * TTM_BK * JT * sizeof(double));
    const int t = threadIdx.x;
    pdl_wait();
    const int64_t p0 = (int64_t)blockIdx.x * TTM_BP;
    const int64_t j0 = (int64_t)blockIdx.y * JT;
    const int64_t ibeg = (int64_t)blockIdx.z * kchunk;
    const int64_t iend = min(I, ibeg + kchunk);
    Y += (int64_t)blockIdx.z * ysize;
    const int64_t nch = (iend - ibeg + TTM_BK - 1) / TTM_BK;
    // ROWS: the CTA's rows are l0..l0+255 of batch b.
    const int64_t b0 = KFAST ? 0 : p0 / L;
    const int64_t l0 = KFAST ? 0 : p0 - b0 * L;
    const TX *xb = KFAST ? X : X + l0 + L * I * b0;

    auto issue = [&](int64_t c, int st) {
        const int64_t i0 = ibeg + c * TTM_BK;
        if (!KFAST) {
            // 16 k x 256 rows: (256 / EV) copies per k.
            constexpr int PER_K = TTM_BP / EV;
            for (int e = t; e < TTM_BK * PER_K; e += TTM_NT) {
                const int k = e / PER_K, q = e - k * PER_K;
                const int64_t i = i0 + k;
                const bool ok = i < iend;
                cp_async16(&Xs[st][k * TTM_BP + q * EV], ok ? xb + L * i + q * EV : X, ok ? 16 : 0);
            }
        } else {
            // 256 rows x 16 i: (16 / EV) copies per row.
            constexpr int PER_R = TTM_BK / EV;
            for (int e = t; e < TTM_BP * PER_R; e += TTM_NT) {
                const int r = e / PER_R, q = e - r * PER_R;
                const int64_t p = p0 + r, i = i0 + q * EV;
                const bool ok = p < P && i < iend;
                cp_async16(&Xs[st][r * KROW + q * EV], ok ? X + p * I + i : X, ok ? 16 : 0);
            }
        }
        for (int e = t; e < TTM_BK * JT; e += TTM_NT) {
            const int k = e / JT, j = e - k * JT;
            const int64_t i = i0 + k, jj = j0 + j;
            const bool ok = i < iend && jj < J;
            cp_async8(&Ms[st][k][j], ok ? M + jj * msj + i * msi : M, ok ? 8 : 0);
        }
        cp_async_commit();
    };

    double acc[2][JT];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int j = 0; j < JT; j++) acc[r][j] = 0.0;

    if (nch > 0) issue(0, 0);
    for (int64_t c = 0; c < nch; c++) {
        const int st = (int)(c & 1);
        if (c + 1 < nch) {
            issue(c + 1, st ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (!KFAST) {
#pragma unroll
            for (int k = 0; k < TTM_BK; k++) {
                double x0, x1;
                if (sizeof(TX) == 4) {
                    const float2 v = *reinterpret_cast<const float2 *>(&Xs[st][k * TTM_BP + 2 * t]);
                    x0 = v.x;
                    x1 = v.y;
                } else {
                    const double2 v = *reinterpret_cast<const double2 *>(&Xs[st][k * TTM_BP + 2 * t]);
                    x0 = v.x;
                    x1 = v.y;
                }
#pragma unroll
                for (int j = 0; j < JT; j += 2) {
                    const double2 m = *reinterpret_cast<const double2 *>(&Ms[st][k][j]);
                    acc[0][j] = fma(x0, m.x, acc[0][j]);
                    acc[0][j + 1] = fma(x0, m.y, acc[0][j + 1]);
                    acc[1][j] = fma(x1, m.x, acc[1][j]);
                    acc[1][j + 1] = fma(x1, m.y, acc[1][j + 1]);
                }
            }
        } else {
            // Rows t and t + 128; EV consecutive k per 16-byte shared load.
#pragma unroll
            for (int kq = 0; kq < TTM_BK; kq += EV) {
                double xv[2][EV];
#pragma unroll
                for (int r = 0; r < 2; r++) {
                    const TX *src = &Xs[st][(t + r * TTM_NT) * KROW + kq];
                    if (sizeof(TX) == 4) {
                        const float4 v = *reinterpret_cast<const float4 *>(src);
                        const float f[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                        for (int q = 0; q < EV; q++) xv[r][q] = f[q];
                    } else {
                        const double2 v = *reinterpret_cast<const double2 *>(src);
                        const double f[2] = {v.x, v.y};
#pragma unroll
                        for (int q = 0; q < EV; q++) xv[r][q] = f[q];
                    }
                }
#pragma unroll
                for (int q = 0; q < EV; q++) {
#pragma unroll
                    for (int j = 0; j < JT; j += 2) {
                        const double2 m = *reinterpret_cast<const double2 *>(&Ms[st][kq + q][j]);
                        acc[0][j] = fma(xv[0][q], m.x, acc[0][j]);
                        acc[0][j + 1] = fma(xv[0][q], m.y, acc[0][j + 1]);
                        acc[1][j] = fma(xv[1][q], m.x, acc[1][j]);
                        acc[1][j + 1] = fma(xv[1][q], m.y, acc[1][j + 1]);
                    }
                }
            }
        }
        __syncthreads();
    }

    pdl_trigger();  // dependents may launch while the outputs are stored
    const int64_t LJ = L * J;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int64_t p = KFAST ? p0 + t + r * TTM_NT : p0 + 2 * t + r;
        if (p >= P) continue;
        const int64_t b = p / L, l = p - b * L;
        double *y = Y + l + LJ * b;
#pragma unroll
        for (int j = 0; j < JT; j++)
            if (j0 + j < J) y[L * (j0 + j)] = acc[r][j];
    }
}

// The ROWS layout on the FP64 tensor cores (mma.sync m8n8k4 .f64), J tile 16.
// The CTA's 256 rows and 16 k of X (and the 16 x 16 slice of M) are staged as
// in ttm_pipe_kernel; warp w owns rows 64 w .. 64 w + 63 as 8 x 2 tiles of 8 x 8
// accumulators.  Per 4-k step a lane converts its 8 A elements (row g of each
// tile, k = t) to FP64 and reads its 2 B elements; 16 mma.sync follow.  The
// staged rows are padded by 32 bytes (X) and the M rows are 20 doubles apart,
// so the four k-rows of a fragment load fall in different banks (64-bit loads
// are served per half-warp).
__device__ __forceinline__ void ttm_dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <class TX>
__host__ __device__ constexpr int ttm_dm_xrow() { return TTM_BP + 32 / (int)sizeof(TX); }  // staged X row pitch
constexpr int TTM_DM_MROW = 20;                                         // staged M row pitch

template <class TX>
__global__ void __launch_bounds__(TTM_NT) ttm_dmma_kernel(const TX *__restrict__ X, int64_t L,
                                                          int64_t I, int64_t P,
                                                          const double *__restrict__ M,
                                                          int64_t msj, int64_t msi, int64_t J,
                                                          double *__restrict__ Y, int64_t kchunk,
                                                          int64_t ysize) {
    constexpr int EV = 16 / sizeof(TX);
    constexpr int TTM_DM_XROW = ttm_dm_xrow<TX>();
    extern __shared__ __align__(16) uint8_t dm_smem[];
    auto Ms = reinterpret_cast<double(*)[TTM_BK * TTM_DM_MROW]>(dm_smem);
    auto Xs = reinterpret_cast<TX(*)[TTM_BK * TTM_DM_XROW]>(
        dm_smem + 2 * TTM_BK * TTM_DM_MROW * sizeof(double));
    const int t = threadIdx.x, w = t >> 5, lane = t & 31, g = lane >> 2, t4 = lane & 3;
    pdl_wait();
    const int64_t p0 = (int64_t)blockIdx.x * TTM_BP;
    const int64_t j0 = (int64_t)blockIdx.y * 16;
    const int64_t ibeg = (int64_t)blockIdx.z * kchunk;
    const int64_t iend = min(I, ibeg + kchunk);
    Y += (int64_t)blockIdx.z * ysize;
    const int64_t nch = (iend - ibeg + TTM_BK - 1) / TTM_BK;
    const int64_t b0 = p0 / L;
    const int64_t l0 = p0 - b0 * L;
    const TX *xb = X + l0 + L * I * b0;

    auto issue = [&](int64_t c, int st) {
        const int64_t i0 = ibeg + c * TTM_BK;
        constexpr int PER_K = TTM_BP / EV;
        for (int e = t; e < TTM_BK * PER_K; e += TTM_NT) {
            const int k = e / PER_K, q = e - k * PER_K;
            const int64_t i = i0 + k;
            const bool ok = i < iend;
            cp_async16(&Xs[st][k * TTM_DM_XROW + q * EV], ok ? xb + L * i + q * EV : X, ok ? 16 : 0);
        }
        for (int e = t; e < TTM_BK * 16; e += TTM_NT) {
            const int k = e >> 4, j = e & 15;
            const int64_t i = i0 + k, jj = j0 + j;
            const bool ok = i < iend && jj < J;
            cp_async8(&Ms[st][k * TTM_DM_MROW + j], ok ? M + jj * msj + i * msi : M, ok ? 8 : 0);
        }
        cp_async_commit();
    };

    double acc[8][2][2];
#pragma unroll
    for (int m = 0; m < 8; m++)
#pragma unroll
        for (int n = 0; n < 2; n++) acc[m][n][0] = acc[m][n][1] = 0.0;

    if (nch > 0) issue(0, 0);
    for (int64_t c = 0; c < nch; c++) {
        const int st = (int)(c & 1);
        if (c + 1 < nch) {
            issue(c + 1, st ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TTM_BK / 4; kk++) {
            const int k = 4 * kk + t4;
            const double b0v = Ms[st][k * TTM_DM_MROW + g];
            const double b1v = Ms[st][k * TTM_DM_MROW + 8 + g];
            const TX *xr = &Xs[st][k * TTM_DM_XROW + 64 * w + g];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const double a = (double)xr[8 * m];
                ttm_dmma884(acc[m][0][0], acc[m][0][1], a, b0v);
                ttm_dmma884(acc[m][1][0], acc[m][1][1], a, b1v);
            }
        }
        __syncthreads();
    }

    pdl_trigger();  // dependents may launch while the outputs are stored
    // D[row g][col 2 t + h] of tile (m, n): row 64 w + 8 m + g, j = 8 n + 2 t + h.
    double *y = Y + l0 + L * J * b0;
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const int64_t row = 64 * w + 8 * m + g;
#pragma unroll
        for (int n = 0; n < 2; n++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int64_t j = j0 + 8 * n + 2 * t4 + h;
                if (j < J) y[row + L * j] = acc[m][n][h];
            }
    }
}

__global__ void sum_splits_kernel(const double *__restrict__ part, int nsplit, int64_t n,
                                  double *__restrict__ out) {
    pdl_wait();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < nsplit; z++) s += part[z * n + e];
        out[e] = s;
    }
    pdl_trigger();
}

template <class TX, int JT>
void ttm_launch(dt_ctx *ctx, const TX *X, int64_t L, int64_t I, int64_t B, const double *M,
                int64_t msj, int64_t msi, int64_t J, double *Y) {
    const int64_t P = L * B;
    const int64_t base = (int64_t)ceil_div(P, TTM_BP) * ceil_div(J, JT);
    // Few output rows: split the contraction so the GPU has enough CTAs, and
    // sum the partial outputs in a fixed order (deterministic).
    int64_t nsplit = 1;
    const int64_t target = 4LL * ctx->num_sms;
    if (base < target && I >= 64) {
        nsplit = std::min<int64_t>((target + base - 1) / base, I / 32);
        nsplit = std::max<int64_t>(nsplit, 1);
    }
    int64_t kchunk = ((I + nsplit - 1) / nsplit + TTM_BK - 1) / TTM_BK * TTM_BK;
    nsplit = (I + kchunk - 1) / kchunk;
    const int64_t ysize = P * J;
    dim3 grid(ceil_div(P, TTM_BP), ceil_div(J, JT), (unsigned)nsplit);
    const uintptr_t xa = reinterpret_cast<uintptr_t>(X);
    const bool rows_ok = L % TTM_BP == 0 && xa % 16 == 0;
    const bool kfast_ok = L == 1 && (I * sizeof(TX)) % 16 == 0 && xa % 16 == 0 &&
                          (kchunk * sizeof(TX)) % 16 == 0;
    constexpr int EV = 16 / sizeof(TX);
    const size_t smem_rows = 2 * TTM_BK * JT * sizeof(double) + 2 * TTM_BK * TTM_BP * sizeof(TX);
    const size_t smem_kfast =
        2 * TTM_BK * JT * sizeof(double) + 2 * TTM_BP * (TTM_BK + EV) * sizeof(TX);
    const size_t smem_dmma = 2 * TTM_BK * TTM_DM_MROW * sizeof(double) +
                             2 * TTM_BK * ttm_dm_xrow<TX>() * sizeof(TX);
    auto launch = [&](double *dst) {
        if (JT == 16 && rows_ok) {
            smem_limit(ctx, ttm_dmma_kernel<TX>, smem_dmma);
            DT_LAUNCH_PDL(ctx, ttm_dmma_kernel<TX>, grid, TTM_NT, smem_dmma, X, L, I, P, M, msj, msi,
                      J, dst, kchunk, ysize);
        } else if (rows_ok) {
            smem_limit(ctx, ttm_pipe_kernel<TX, JT, false>, smem_rows);
            DT_LAUNCH_PDL(ctx, (ttm_pipe_kernel<TX, JT, false>), grid, TTM_NT, smem_rows, X, L, I, P,
                      M, msj, msi, J, dst, kchunk, ysize);
        } else if (kfast_ok) {
            smem_limit(ctx, ttm_pipe_kernel<TX, JT, true>, smem_kfast);
            DT_LAUNCH_PDL(ctx, (ttm_pipe_kernel<TX, JT, true>), grid, TTM_NT, smem_kfast, X, L, I, P,
                      M, msj, msi, J, dst, kchunk, ysize);
        }
        else
            DT_LAUNCH_PDL(ctx, (ttm_kernel<TX, JT>), grid, TTM_NT, 0, X, L, I, P, M, msj, msi, J, dst,
                      kchunk, ysize);
    };
    if (nsplit == 1) {
        launch(Y);
        return;
    }
    DevMem part(ctx, (size_t)nsplit * ysize * sizeof(double));
    launch(part.as<double>());
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceil_div(ysize, 256), 8u * ctx->num_sms));
    DT_LAUNCH_PDL(ctx, sum_splits_kernel, blocks, 256, 0, part.as<double>(), (int)nsplit, ysize, Y);
}

}  // namespace

template <class TX>
void ttm_f64(dt_ctx *ctx, const TX *X, int64_t L, int64_t I, int64_t B, const double *M,
             int64_t msj, int64_t msi, int64_t J, double *Y) {
    if (L * B == 0 || J == 0) return;
    if (J <= 4)
        ttm_launch<TX, 4>(ctx, X, L, I, B, M, msj, msi, J, Y);
    else if (J <= 8)
        ttm_launch<TX, 8>(ctx, X, L, I, B, M, msj, msi, J, Y);
    else
        ttm_launch<TX, 16>(ctx, X, L, I, B, M, msj, msi, J, Y);
}
template void ttm_f64<double>(dt_ctx *, const double *, int64_t, int64_t, int64_t,
                              const double *, int64_t, int64_t, int64_t, double *);
template void ttm_f64<float>(dt_ctx *, const float *, int64_t, int64_t, int64_t,
                             const double *, int64_t, int64_t, int64_t, double *);

// ---------------------------------------------------------------------------
// Generic FP64 GEMM C(i, j) = sum_q a(i, q) b(j, q) over operands addressed as
//   a(i, q) = A[koff(q) + i * si],  koff(q) = q * sk            (plain matrix)
//                                   koff(q) = (q % L) + LI*(q / L)  (unfolding)
// This covers Function::gram / ttt_except (both operands are mode-n
// unfoldings X_(n), q running over the other modes) and matmulNN/NT/TN.
// 64 x 64 output tiles on the FP64 tensor cores, split-K over gridDim.z with
// a deterministic reduction of the partial tiles.
// ---------------------------------------------------------------------------
namespace {

struct Operand {
    const double *p;
    int64_t si;   // stride of the output index (i or j)
    int64_t sk;   // stride of q for a plain matrix
    int64_t L;    // unfolding: run length of q with unit stride
    int64_t LI;   // unfolding: stride of q / L
    int unfold;
    int kfast;    // consecutive q are adjacent in memory
};

__device__ __forceinline__ int64_t koff(const Operand &o, int64_t q) {
    if (o.unfold) {
        const int64_t b = q / o.L;
        return (q - b * o.L) + o.LI * b;
    }
    return q * o.sk;
}

constexpr int GM_B = 64;
constexpr int GM_BK = 16;
constexpr int GM_NT = 256;
// Staged rows are 68 doubles apart: the four k-rows of an mma.sync fragment
// load (lanes g + 8 t, 64-bit loads served per half-warp) fall in different
// banks.
constexpr int GM_P = GM_B + 4;

// One thread's four elements of a 16 x 64 operand tile: fetched into
// registers (fetch) while the previous tile is consumed, then stored (store).
struct TileRegs {
    double v[4];
};

__device__ __forceinline__ void fetch_tile(TileRegs &r, const Operand &o, int64_t i0, int64_t nI,
                                           int64_t q0, int64_t qend, int t) {
    if (o.kfast) {
        // 16 consecutive q per row, 16 rows per pass.
        const int k = t & 15;
        const int64_t q = q0 + k;
        const bool qok = q < qend;
        const int64_t off = qok ? koff(o, q) : 0;
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const int64_t i = i0 + (t >> 4) + 16 * s;
            r.v[s] = (qok && i < nI) ? o.p[off + i * o.si] : 0.0;
        }
    } else {
        // 64 consecutive output indices per q, 4 q per pass.
        const int64_t i = i0 + (t & 63);
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const int64_t q = q0 + (t >> 6) + 4 * s;
            r.v[s] = (q < qend && i < nI) ? o.p[koff(o, q) + i * o.si] : 0.0;
        }
    }
}

__device__ __forceinline__ void store_tile(double (*dst)[GM_P], const TileRegs &r,
                                           const Operand &o, int t) {
    if (o.kfast) {
#pragma unroll
        for (int s = 0; s < 4; s++) dst[t & 15][(t >> 4) + 16 * s] = r.v[s];
    } else {
#pragma unroll
        for (int s = 0; s < 4; s++) dst[(t >> 6) + 4 * s][t & 63] = r.v[s];
    }
}

__device__ __forceinline__ void gm_dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// 64 x 64 output tile per CTA on the FP64 tensor cores (mma.sync m8n8k4):
// warp w owns rows 32 (w % 2) .. + 31 and columns 16 (w / 2) .. + 15 as 4 x 2
// tiles of 8 x 8.  Lane (g, t) supplies a(row g, q = t) and b(col g, q = t)
// and holds D[row g][cols 2 t, 2 t + 1].  The next 16 q of both operands are
// fetched into registers while the current ones are multiplied.
__global__ void __launch_bounds__(GM_NT) gemm_kernel(Operand A, Operand B, int64_t M,
                                                     int64_t N, int64_t K, int64_t kchunk,
                                                     double *__restrict__ C, int64_t ldc,
                                                     double beta, double *__restrict__ part) {
    __shared__ __align__(16) double As[GM_BK][GM_P];
    __shared__ __align__(16) double Bs[GM_BK][GM_P];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31, g = lane >> 2, t4 = lane & 3;
    const int rb = 32 * (w & 1), cb = 16 * (w >> 1);
    const int64_t i0 = (int64_t)blockIdx.x * GM_B;
    const int64_t j0 = (int64_t)blockIdx.y * GM_B;
    const int64_t qbeg = (int64_t)blockIdx.z * kchunk;
    const int64_t qend = min(K, qbeg + kchunk);
    double acc[4][2][2];
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
        for (int n = 0; n < 2; n++) acc[m][n][0] = acc[m][n][1] = 0.0;
    TileRegs ra, rb_;
    if (qbeg < qend) {
        fetch_tile(ra, A, i0, M, qbeg, qend, t);
        fetch_tile(rb_, B, j0, N, qbeg, qend, t);
    }
    for (int64_t q0 = qbeg; q0 < qend; q0 += GM_BK) {
        store_tile(As, ra, A, t);
        store_tile(Bs, rb_, B, t);
        __syncthreads();
        if (q0 + GM_BK < qend) {
            fetch_tile(ra, A, i0, M, q0 + GM_BK, qend, t);
            fetch_tile(rb_, B, j0, N, q0 + GM_BK, qend, t);
        }
#pragma unroll
        for (int kk = 0; kk < GM_BK / 4; kk++) {
            const int k = 4 * kk + t4;
            const double b0 = Bs[k][cb + g], b1 = Bs[k][cb + 8 + g];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const double a = As[k][rb + 8 * m + g];
                gm_dmma884(acc[m][0][0], acc[m][0][1], a, b0);
                gm_dmma884(acc[m][1][0], acc[m][1][1], a, b1);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int64_t i = i0 + rb + 8 * m + g;
        if (i >= M) continue;
#pragma unroll
        for (int n = 0; n < 2; n++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int64_t j = j0 + cb + 8 * n + 2 * t4 + h;
                if (j >= N) continue;
                if (part)
                    part[(int64_t)blockIdx.z * M * N + i + M * j] = acc[m][n][h];
                else
                    C[i + ldc * j] = acc[m][n][h] + (beta != 0.0 ? beta * C[i + ldc * j] : 0.0);
            }
    }
}

__global__ void splitk_reduce_kernel(const double *__restrict__ part, int nsplit, int64_t M,
                                     int64_t N, double *__restrict__ C, int64_t ldc,
                                     double beta) {
    const int64_t MN = M * N;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < MN;
         e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < nsplit; z++) s += part[z * MN + e];
        const int64_t i = e % M, j = e / M;
        C[i + ldc * j] = s + (beta != 0.0 ? beta * C[i + ldc * j] : 0.0);
    }
}

void gemm_generic(dt_ctx *ctx, const Operand &A, const Operand &B, int64_t M, int64_t N,
                  int64_t K, double *C, int64_t ldc, double beta) {
    if (M == 0 || N == 0) return;
    const int64_t tiles = (int64_t)ceil_div(M, GM_B) * ceil_div(N, GM_B);
    const int64_t target = 2LL * ctx->num_sms;
    int64_t nsplit = 1;
    if (tiles < target && K > 256) {
        nsplit = (target + tiles - 1) / tiles;
        nsplit = std::min<int64_t>(nsplit, (K + 127) / 128);
        nsplit = std::max<int64_t>(nsplit, 1);
    }
    int64_t kchunk = (K + nsplit - 1) / nsplit;
    kchunk = ((kchunk + GM_BK - 1) / GM_BK) * GM_BK;
    if (kchunk == 0) kchunk = GM_BK;
    nsplit = (K + kchunk - 1) / kchunk;
    if (nsplit < 1) nsplit = 1;
    dim3 grid(ceil_div(M, GM_B), ceil_div(N, GM_B), (unsigned)nsplit);
    if (nsplit == 1) {
        DT_LAUNCH(ctx, gemm_kernel, grid, GM_NT, 0, A, B, M, N, K, kchunk, C, ldc, beta,
                  (double *)nullptr);
    } else {
        DevMem part(ctx, (size_t)nsplit * M * N * sizeof(double));
        DT_LAUNCH(ctx, gemm_kernel, grid, GM_NT, 0, A, B, M, N, K, kchunk, C, ldc, beta,
                  part.as<double>());
        const unsigned blocks = std::min<unsigned>(ceil_div(M * N, 256), 4096u);
        DT_LAUNCH(ctx, splitk_reduce_kernel, blocks, 256, 0, part.as<double>(), (int)nsplit, M,
                  N, C, ldc, beta);
    }
}

Operand plain(const double *p, int64_t si, int64_t sk) {
    Operand o{p, si, sk, 1, 0, 0, sk == 1 ? 1 : 0};
    return o;
}

Operand unfolding(const double *p, int64_t L, int64_t I) {
    Operand o{p, L, 0, L, L * I, 1, L >= 16 ? 1 : 0};
    return o;
}

}  // namespace

void ttt_f64(dt_ctx *ctx, const double *A, const double *Bt, int64_t L, int64_t IA,
             int64_t IB, int64_t B, double *C) {
    gemm_generic(ctx, unfolding(A, L, IA), unfolding(Bt, L, IB), IA, IB, L * B, C, IA, 0.0);
}

void ttt_f64_scratch(dt_ctx *ctx, const double *A, const double *Bt, int64_t L, int64_t IA,
                     int64_t IB, int64_t B, double *C, double *scratch, int64_t scratch_doubles) {
    // Same tiles, split choice and reduction as gemm_generic, with the split-K
    // partial tiles in the caller's scratch; the split count is lowered when
    // nsplit * IA * IB doubles would not fit.
    const int64_t M = IA, N = IB, K = L * B;
    if (M == 0 || N == 0) return;
    const int64_t MN = M * N;
    DT_CHECK_ARG(MN <= scratch_doubles,
                 "ttt_f64_scratch: %lld x %lld result needs more than %lld scratch doubles",
                 (long long)M, (long long)N, (long long)scratch_doubles);
    const Operand a = unfolding(A, L, IA), b = unfolding(Bt, L, IB);
    const int64_t tiles = (int64_t)ceil_div(M, GM_B) * ceil_div(N, GM_B);
    const int64_t target = 2LL * ctx->num_sms;
    int64_t nsplit = 1;
    if (tiles < target && K > 256) {
        nsplit = (target + tiles - 1) / tiles;
        nsplit = std::min<int64_t>(nsplit, (K + 127) / 128);
        nsplit = std::min<int64_t>(nsplit, scratch_doubles / MN);
        nsplit = std::max<int64_t>(nsplit, 1);
    }
    int64_t kchunk = (K + nsplit - 1) / nsplit;
    kchunk = ((kchunk + GM_BK - 1) / GM_BK) * GM_BK;
    if (kchunk == 0) kchunk = GM_BK;
    nsplit = (K + kchunk - 1) / kchunk;
    if (nsplit < 1) nsplit = 1;
    dim3 grid(ceil_div(M, GM_B), ceil_div(N, GM_B), (unsigned)nsplit);
    if (nsplit == 1) {
        DT_LAUNCH(ctx, gemm_kernel, grid, GM_NT, 0, a, b, M, N, K, kchunk, C, M, 0.0,
                  (double *)nullptr);
    } else {
        DT_LAUNCH(ctx, gemm_kernel, grid, GM_NT, 0, a, b, M, N, K, kchunk, C, M, 0.0, scratch);
        const unsigned blocks = std::min<unsigned>(ceil_div(MN, 256), 4096u);
        DT_LAUNCH(ctx, splitk_reduce_kernel, blocks, 256, 0, (const double *)scratch, (int)nsplit,
                  M, N, C, M, 0.0);
    }
}

void gemm_f64(dt_ctx *ctx, int transA, int transB, int64_t m, int64_t n, int64_t k,
              const double *A, int64_t lda, const double *B, int64_t ldb, double *C,
              int64_t ldc, double beta) {
    // a(i, q) = op(A)(i, q); b(j, q) = op(B)(q, j).
    const Operand a = transA ? plain(A, lda, 1) : plain(A, 1, lda);
    const Operand b = transB ? plain(B, 1, ldb) : plain(B, ldb, 1);
    gemm_generic(ctx, a, b, m, n, k, C, ldc, beta);
}

// ---------------------------------------------------------------------------
// Norms and conversions.
// ---------------------------------------------------------------------------
namespace {

template <class T>
__global__ void sumsq_partial_kernel(const T *__restrict__ x, int64_t n,
                                     double *__restrict__ part) {
    pdl_wait();
    double s = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)x[e];
        s = fma(v, v, s);
    }
    pdl_trigger();
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) part[blockIdx.x] = s;
    }
}

__global__ void sum_partials_kernel(const double *__restrict__ part, int n,
                                    double *__restrict__ out) {
    pdl_wait();
    double s = 0.0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) s += part[e];
    pdl_trigger();
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) out[0] = s;
    }
}

__global__ void f32_to_f64_kernel(const float *__restrict__ x, int64_t n,
                                  double *__restrict__ y) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        y[e] = (double)x[e];
}

}  // namespace

void sumsq(dt_ctx *ctx, const void *x, int dtype, int64_t n, double *out) {
    const int blocks = std::max(1, std::min<int>(4 * ctx->num_sms, (int)ceil_div(n, 256)));
    DevMem part(ctx, (size_t)blocks * sizeof(double));
    if (dtype == DT_F64)
        DT_LAUNCH_PDL(ctx, sumsq_partial_kernel<double>, blocks, 256, 0,
                  static_cast<const double *>(x), n, part.as<double>());
    else
        DT_LAUNCH_PDL(ctx, sumsq_partial_kernel<float>, blocks, 256, 0,
                  static_cast<const float *>(x), n, part.as<double>());
    DT_LAUNCH_PDL(ctx, sum_partials_kernel, 1, 1024, 0, part.as<double>(), blocks, out);
}

void f32_to_f64(dt_ctx *ctx, const float *x, int64_t n, double *y) {
    const int blocks = std::max(1, std::min<int>(8 * ctx->num_sms, (int)ceil_div(n, 256)));
    DT_LAUNCH(ctx, f32_to_f64_kernel, blocks, 256, 0, x, n, y);
}

}  // namespace dt
