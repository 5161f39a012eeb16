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
                                                     double *__restrict__ Y) {
    __shared__ __align__(16) double Xs[TTM_BK][TTM_BP];
    __shared__ __align__(16) double Ms[TTM_BK][JT];
    const int t = threadIdx.x;
    const int64_t p0 = (int64_t)blockIdx.x * TTM_BP;
    const int64_t j0 = (int64_t)blockIdx.y * JT;
    const int64_t LI = L * I;

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

    for (int64_t i0 = 0; i0 < I; i0 += TTM_BK) {
        if (L > 1) {
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int pp = t + s * TTM_NT;
#pragma unroll 4
                for (int k = 0; k < TTM_BK; k++) {
                    const int64_t i = i0 + k;
                    Xs[k][pp] = (lok[s] && i < I) ? (double)X[lbase[s] + L * i] : 0.0;
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
                Xs[k][pp] = (p < P && i < I) ? (double)X[p * I + i] : 0.0;
            }
        }
        for (int e = t; e < TTM_BK * JT; e += TTM_NT) {
            const int k = e / JT, j = e - (e / JT) * JT;
            const int64_t i = i0 + k, jj = j0 + j;
            Ms[k][j] = (i < I && jj < J) ? M[jj * msj + i * msi] : 0.0;
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

template <class TX, int JT>
void ttm_launch(dt_ctx *ctx, const TX *X, int64_t L, int64_t I, int64_t B, const double *M,
                int64_t msj, int64_t msi, int64_t J, double *Y) {
    const int64_t P = L * B;
    dim3 grid(ceil_div(P, TTM_BP), ceil_div(J, JT));
    DT_LAUNCH(ctx, (ttm_kernel<TX, JT>), grid, TTM_NT, 0, X, L, I, P, M, msj, msi, J, Y);
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
// 64 x 64 output tiles, 4 x 4 per thread, split-K over gridDim.z with a
// deterministic reduction of the partial tiles.
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

__device__ __forceinline__ void load_tile(double (*dst)[GM_B], const Operand &o, int64_t i0,
                                          int64_t nI, int64_t q0, int64_t qend, int t) {
    if (o.kfast) {
        // 16 consecutive q per row, 16 rows per pass.
        const int k = t & 15;
        const int64_t q = q0 + k;
        const bool qok = q < qend;
        const int64_t off = qok ? koff(o, q) : 0;
#pragma unroll
        for (int s = 0; s < GM_B / 16; s++) {
            const int m = (t >> 4) + 16 * s;
            const int64_t i = i0 + m;
            dst[k][m] = (qok && i < nI) ? o.p[off + i * o.si] : 0.0;
        }
    } else {
        // 64 consecutive output indices per q, 4 q per pass.
        const int m = t & 63;
        const int64_t i = i0 + m;
#pragma unroll
        for (int s = 0; s < GM_BK / 4; s++) {
            const int k = (t >> 6) + 4 * s;
            const int64_t q = q0 + k;
            dst[k][m] = (q < qend && i < nI) ? o.p[koff(o, q) + i * o.si] : 0.0;
        }
    }
}

__global__ void __launch_bounds__(GM_NT) gemm_kernel(Operand A, Operand B, int64_t M,
                                                     int64_t N, int64_t K, int64_t kchunk,
                                                     double *__restrict__ C, int64_t ldc,
                                                     double beta, double *__restrict__ part) {
    __shared__ __align__(16) double As[GM_BK][GM_B];
    __shared__ __align__(16) double Bs[GM_BK][GM_B];
    const int t = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * GM_B;
    const int64_t j0 = (int64_t)blockIdx.y * GM_B;
    const int64_t qbeg = (int64_t)blockIdx.z * kchunk;
    const int64_t qend = min(K, qbeg + kchunk);
    const int tx = t & 15, ty = t >> 4;
    double acc[4][4] = {};
    for (int64_t q0 = qbeg; q0 < qend; q0 += GM_BK) {
        load_tile(As, A, i0, M, q0, qend, t);
        load_tile(Bs, B, j0, N, q0, qend, t);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < GM_BK; k++) {
            const double2 a01 = *reinterpret_cast<const double2 *>(&As[k][4 * tx]);
            const double2 a23 = *reinterpret_cast<const double2 *>(&As[k][4 * tx + 2]);
            const double2 b01 = *reinterpret_cast<const double2 *>(&Bs[k][4 * ty]);
            const double2 b23 = *reinterpret_cast<const double2 *>(&Bs[k][4 * ty + 2]);
            const double a[4] = {a01.x, a01.y, a23.x, a23.y};
            const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int64_t i = i0 + 4 * tx + u;
        if (i >= M) continue;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int64_t j = j0 + 4 * ty + v;
            if (j >= N) continue;
            if (part)
                part[(int64_t)blockIdx.z * M * N + i + M * j] = acc[u][v];
            else
                C[i + ldc * j] = acc[u][v] + (beta != 0.0 ? beta * C[i + ldc * j] : 0.0);
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
    double s = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)x[e];
        s = fma(v, v, s);
    }
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
    double s = 0.0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) s += part[e];
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
        DT_LAUNCH(ctx, sumsq_partial_kernel<double>, blocks, 256, 0,
                  static_cast<const double *>(x), n, part.as<double>());
    else
        DT_LAUNCH(ctx, sumsq_partial_kernel<float>, blocks, 256, 0,
                  static_cast<const float *>(x), n, part.as<double>());
    DT_LAUNCH(ctx, sum_partials_kernel, 1, 1024, 0, part.as<double>(), blocks, out);
}

void f32_to_f64(dt_ctx *ctx, const float *x, int64_t n, double *y) {
    const int blocks = std::max(1, std::min<int>(8 * ctx->num_sms, (int)ceil_div(n, 256)));
    DT_LAUNCH(ctx, f32_to_f64_kernel, blocks, 256, 0, x, n, y);
}

}  // namespace dt
