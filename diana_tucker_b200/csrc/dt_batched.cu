// Batched dense HOOI: many small 3-way tensors of uneven shapes and ranks
// decomposed in one persistent launch.
//
// Work items.  The host sorts the tensors by estimated cost (longest first,
// so the persistent CTAs finish together) and packs them into items: an item
// is one tensor worked on by the whole CTA, or two or four small tensors
// worked on side by side by equal thread groups of the CTA (each group with
// its own named barrier, its own slice of shared memory and of the global
// scratch).  Each CTA pulls items from an atomic queue.
//
// Per tensor, the whole HOOI runs inside its thread group: the
// dimension-tree TTM chain (T = X x_3 U_3^T shared by modes 1 and 2,
// X x_1 U_1^T x_2 U_2^T for mode 3), the Gram Y_(n) Y_(n)^T, the subspace
// iteration of ALS_ (hooi_als.tpp:7-34) with CholeskyQR, and finally the FP64
// core and relative error.  X is read from global memory (mostly from L2 while
// its group works on it), Y_(n), the Gram and the factors live in shared
// memory, the one large intermediate (I_1 x I_2 x R_3) in the group's slice of
// global scratch.  Arithmetic is FP64 throughout; X is FP32.  The reductions
// keep four independent FMA chains per thread (the FP64 FMA latency is ~23
// cycles), in a fixed order, so results do not depend on the launch shape.
//
// Autotuning.  The block size (128, 256, 512 threads) and the packing (one
// tensor per CTA; pairs, and quads, of the tensors small enough to share the
// CTA's shared memory: largest mode <= 37, <= 21) are chosen by timing every
// combination on the batch (a stratified sample of 8192 tensors of larger
// batches); the choice is cached per batch signature on the context.
//
// The launch (queue reset + persistent kernel) is a CUDA graph instantiated
// once per launch shape and kept on the context: the kernel reads its
// arguments from a device-resident block that each call rewrites, so a later
// call with the same launch shape replays the graph without re-capturing.
// On the legacy or per-thread default stream, which cannot be captured, the
// two are launched directly.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>
#include <vector>

#include "dt_kernels.cuh"

namespace dt {
namespace {

constexpr int BMAX_I = 64;               // largest mode size
constexpr int BMAX_R = 8;                // largest rank
constexpr int BMAX_K = BMAX_R * BMAX_R;  // largest product of two ranks

// Shared-memory doubles one tensor of largest mode size m needs:
// U (3 m R), Y (m K), S (m^2), Z (m R), the R x R Gram, reduction scratch.
__host__ __device__ constexpr int slot_doubles(int m) {
    return 3 * m * BMAX_R + m * BMAX_K + m * m + m * BMAX_R + BMAX_R * BMAX_R + 40;
}
constexpr int SLOT = slot_doubles(BMAX_I);                    // one CTA
constexpr int64_t SCR = (int64_t)BMAX_I * BMAX_I * BMAX_R;    // global scratch per CTA
// Largest mode size a tensor may have to share a CTA with 1 / 3 others: its
// shared-memory needs fit SLOT / g (its scratch then fits SCR / g as well).
constexpr int pack_limit(int g) {
    int m = BMAX_I;
    while (m > 0 && slot_doubles(m) > SLOT / g) m--;
    return m;
}
constexpr int PAIR_MAX_I = pack_limit(2);  // 37
constexpr int QUAD_MAX_I = pack_limit(4);  // 21
static_assert(PAIR_MAX_I == 37 && QUAD_MAX_I == 21, "packing limits");
static_assert((int64_t)PAIR_MAX_I * PAIR_MAX_I * BMAX_R <= SCR / 2, "pair scratch");
static_assert((int64_t)QUAD_MAX_I * QUAD_MAX_I * BMAX_R <= SCR / 4, "quad scratch");

struct Item {
    int g;     // tensors worked on side by side (1, 2 or 4)
    int t[4];  // tensor ids, -1 where a group has none
};

struct BatchArgs {
    int count, nitems;
    const int64_t *shape;  // count x 3
    const int64_t *rank;   // count x 3
    const float *X;
    const int64_t *xoff;   // element offsets of each tensor
    double *U;             // factors, I_n x R_n col-major blocks
    const int64_t *uoff;   // count x 3 element offsets
    double *G;             // cores
    const int64_t *goff;
    double *relerr;
    const Item *items;
    int sweeps, inner;
    double *scratch;       // gridDim.x x SCR doubles
    int *queue;
};

// A thread group working on one tensor: its threads are a contiguous run of
// whole warps of the CTA, synchronised by their own named barrier.
struct Grp {
    int lt;   // thread index in the group
    int gs;   // threads in the group (a multiple of 32)
    int bar;  // named barrier id (1..4; 0 is __syncthreads)
};

__device__ __forceinline__ void gsync(const Grp &g) {
    asm volatile("bar.sync %0, %1;" ::"r"(g.bar), "r"(g.gs) : "memory");
}

// Sum over the group, fixed order (warp tree, then warps in order).
__device__ double gsum(double v, double *red, const Grp &g) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = g.lt >> 5, l = g.lt & 31;
    gsync(g);
    if (l == 0) red[w] = v;
    gsync(g);
    if (g.lt == 0) {
        double s = 0.0;
        for (int i = 0; i < (g.gs >> 5); i++) s += red[i];
        red[32] = s;
    }
    gsync(g);
    const double r = red[32];
    gsync(g);
    return r;
}

// Cholesky of the r x r Gram in G (row-major, r <= 8) by lane c owning column
// c; overwrites G with R (upper).  Returns false on a non-positive pivot.
// Called by one full warp.
__device__ bool warp_chol8(double *G, int r) {
    const int lane = threadIdx.x & 31;
    double g[BMAX_R];
#pragma unroll
    for (int i = 0; i < BMAX_R; i++) g[i] = (i < r && lane < r) ? G[i * r + lane] : 0.0;
    const double g00 = __shfl_sync(0xffffffffu, g[0], 0);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < BMAX_R; k++) {
        if (k >= r) break;
        const double d = __shfl_sync(0xffffffffu, g[k], k);
        if (!(d > 1e-28 * g00)) ok = false;
        const double rkk = sqrt(fmax(d, 1e-300));
        const double inv = 1.0 / rkk;
        if (lane > k) g[k] *= inv;
        if (lane == k) g[k] = rkk;
#pragma unroll
        for (int i = k + 1; i < BMAX_R; i++) {
            if (i >= r) break;
            const double rki = __shfl_sync(0xffffffffu, g[k], i);
            if (lane >= i) g[i] = fma(-rki, g[k], g[i]);
        }
    }
    if (lane < r) {
#pragma unroll
        for (int i = 0; i < BMAX_R; i++)
            if (i < r) G[i * r + lane] = i <= lane ? g[i] : 0.0;
    }
    __syncwarp();
    return ok;
}

// dst (n x r col-major) = orth(src) by CholeskyQR; Gs is r x r scratch.
// Falls back to modified Gram-Schmidt when the Gram is not positive definite.
__device__ void gcholqr(const double *src, double *dst, int n, int r, double *Gs, int *bad,
                        const Grp &g) {
    // The r x r Gram: four threads per entry, each summing every fourth row,
    // combined by two shuffles (a fixed order).
    const int total = 4 * r * r;
    for (int base = 0; base < total; base += g.gs) {
        const int idx = base + g.lt;
        const int e = idx >> 2, part = idx & 3;
        double s = 0.0;
        if (idx < total) {
            const int a = e / r, b = e % r;
            const double *pa = src + a * n, *pb = src + b * n;
            for (int k = part; k < n; k += 4) s = fma(pa[k], pb[k], s);
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (idx < total && part == 0) Gs[e] = s;
    }
    gsync(g);
    if (g.lt < 32) {
        const bool ok = warp_chol8(Gs, r);
        if (g.lt == 0) *bad = ok ? 0 : 1;
    }
    gsync(g);
    if (!*bad) {
        for (int i = g.lt; i < n; i += g.gs) {
            double q[BMAX_R];
#pragma unroll
            for (int c = 0; c < BMAX_R; c++) {
                if (c >= r) break;
                double acc = src[i + c * n];
#pragma unroll
                for (int k = 0; k < BMAX_R; k++) {
                    if (k >= c) break;
                    acc = fma(-q[k], Gs[k * r + c], acc);
                }
                q[c] = acc / Gs[c * r + c];
                dst[i + c * n] = q[c];
            }
        }
        gsync(g);
        return;
    }
    // Rank-deficient product: modified Gram-Schmidt with zero columns kept zero.
    if (g.lt == 0) {
        for (int c = 0; c < r; c++) {
            for (int i = 0; i < n; i++) dst[i + c * n] = src[i + c * n];
            for (int p = 0; p < c; p++) {
                double d = 0.0;
                for (int i = 0; i < n; i++) d += dst[i + c * n] * dst[i + p * n];
                for (int i = 0; i < n; i++) dst[i + c * n] -= d * dst[i + p * n];
            }
            double nr = 0.0;
            for (int i = 0; i < n; i++) nr += dst[i + c * n] * dst[i + c * n];
            nr = sqrt(nr);
            for (int i = 0; i < n; i++) dst[i + c * n] = nr > 0 ? dst[i + c * n] / nr : 0.0;
        }
    }
    gsync(g);
}

// Leading subspace of S (n x n, symmetric) from L (n x r), `iters` steps of
// L <- orth(S L), in place on L.
__device__ void gsubspace(const double *S, int n, double *L, int r, int iters, double *Z,
                          double *Gs, int *bad, const Grp &g) {
    for (int it = 0; it < iters; it++) {
        for (int e = g.lt; e < n * r; e += g.gs) {
            const int i = e % n, c = e / n;
            const double *lc = L + n * c;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            int k = 0;
            for (; k + 3 < n; k += 4) {
                a0 = fma(S[i + n * k], lc[k], a0);
                a1 = fma(S[i + n * (k + 1)], lc[k + 1], a1);
                a2 = fma(S[i + n * (k + 2)], lc[k + 2], a2);
                a3 = fma(S[i + n * (k + 3)], lc[k + 3], a3);
            }
            for (; k < n; k++) a0 = fma(S[i + n * k], lc[k], a0);
            Z[e] = (a0 + a1) + (a2 + a3);
        }
        gsync(g);
        gcholqr(Z, L, n, r, Gs, bad, g);
    }
}

// S (n x n) = Y Y^T for Y n x K col-major (row i at Y[i + n k]): 2 x 2 blocks
// of S per thread, four independent chains.
__device__ void ggram(const double *Y, int n, int K, double *S, const Grp &g) {
    const int nb = (n + 1) >> 1;
    for (int e = g.lt; e < nb * nb; e += g.gs) {
        const int bi = e % nb, bj = e / nb;
        if (bj < bi) continue;  // upper block triangle; mirrored below
        const int i0 = 2 * bi, j0 = 2 * bj;
        const int i1 = min(i0 + 1, n - 1), j1 = min(j0 + 1, n - 1);
        double s00 = 0.0, s01 = 0.0, s10 = 0.0, s11 = 0.0;
        for (int k = 0; k < K; k++) {
            const double *y = Y + n * k;
            const double a0 = y[i0], a1 = y[i1], b0 = y[j0], b1 = y[j1];
            s00 = fma(a0, b0, s00);
            s01 = fma(a0, b1, s01);
            s10 = fma(a1, b0, s10);
            s11 = fma(a1, b1, s11);
        }
        S[i0 + n * j0] = s00;
        S[j0 + n * i0] = s00;
        if (j0 + 1 < n) {
            S[i0 + n * j1] = s01;
            S[j1 + n * i0] = s01;
        }
        if (i0 + 1 < n) {
            S[i1 + n * j0] = s10;
            S[j0 + n * i1] = s10;
        }
        if (i0 + 1 < n && j0 + 1 < n) {
            S[i1 + n * j1] = s11;
            S[j1 + n * i1] = s11;
        }
    }
    gsync(g);
}

// The whole HOOI of tensor t by one thread group.  `sm` is the group's
// shared-memory slice (slot_doubles(largest mode) doubles at least), `T` its
// global scratch slice.
__device__ void hooi_one(const BatchArgs &a, int t, double *sm, double *T, const Grp &g,
                         int *bad) {
    const int I0 = (int)a.shape[3 * t], I1 = (int)a.shape[3 * t + 1], I2 = (int)a.shape[3 * t + 2];
    const int R0 = (int)a.rank[3 * t], R1 = (int)a.rank[3 * t + 1], R2 = (int)a.rank[3 * t + 2];
    const int m = max(I0, max(I1, I2));
    double *U0 = sm, *U1 = U0 + m * BMAX_R, *U2 = U1 + m * BMAX_R;
    double *Ys = U2 + m * BMAX_R;   // m x K
    double *Ss = Ys + m * BMAX_K;   // m x m
    double *Zs = Ss + m * m;        // m x R
    double *Gs = Zs + m * BMAX_R;   // R x R
    double *red = Gs + BMAX_R * BMAX_R;
    const float *X = a.X + a.xoff[t];
    double *ug[3] = {a.U + a.uoff[3 * t], a.U + a.uoff[3 * t + 1], a.U + a.uoff[3 * t + 2]};
    for (int e = g.lt; e < I0 * R0; e += g.gs) U0[e] = ug[0][e];
    for (int e = g.lt; e < I1 * R1; e += g.gs) U1[e] = ug[1][e];
    for (int e = g.lt; e < I2 * R2; e += g.gs) U2[e] = ug[2][e];
    const int64_t nx = (int64_t)I0 * I1 * I2;
    double s = 0.0;
    for (int64_t e = g.lt; e < nx; e += g.gs) s = fma((double)X[e], (double)X[e], s);
    const double x2 = gsum(s, red, g);
    const int I01 = I0 * I1;
    for (int sw = 0; sw < a.sweeps; sw++) {
        // T = X x_3 U_3^T  (I0 x I1 x R2)
        for (int p = g.lt; p < I01; p += g.gs) {
            double acc[BMAX_R] = {};
#pragma unroll 4
            for (int i2 = 0; i2 < I2; i2++) {
                const double x = X[p + (int64_t)I01 * i2];
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R2) acc[r] = fma(x, U2[i2 + I2 * r], acc[r]);
            }
#pragma unroll
            for (int r = 0; r < BMAX_R; r++)
                if (r < R2) T[p + I01 * r] = acc[r];
        }
        gsync(g);
        // Mode 1: Y_(1)[i0, r1 + R1 r2] = sum_i1 T[i0, i1, r2] U1[i1, r1]
        for (int q = g.lt; q < I0 * R2; q += g.gs) {
            const int i0 = q % I0, r2 = q / I0;
            double acc[BMAX_R] = {};
#pragma unroll 4
            for (int i1 = 0; i1 < I1; i1++) {
                const double v = T[i0 + I0 * i1 + I01 * r2];
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R1) acc[r] = fma(v, U1[i1 + I1 * r], acc[r]);
            }
#pragma unroll
            for (int r = 0; r < BMAX_R; r++)
                if (r < R1) Ys[i0 + I0 * (r + R1 * r2)] = acc[r];
        }
        gsync(g);
        ggram(Ys, I0, R1 * R2, Ss, g);
        gsubspace(Ss, I0, U0, R0, a.inner, Zs, Gs, bad, g);
        // Mode 2: Y_(2)[i1, r0 + R0 r2] = sum_i0 T[i0, i1, r2] U0[i0, r0]
        for (int q = g.lt; q < I1 * R2; q += g.gs) {
            const int i1 = q % I1, r2 = q / I1;
            double acc[BMAX_R] = {};
#pragma unroll 4
            for (int i0 = 0; i0 < I0; i0++) {
                const double v = T[i0 + I0 * i1 + I01 * r2];
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R0) acc[r] = fma(v, U0[i0 + I0 * r], acc[r]);
            }
#pragma unroll
            for (int r = 0; r < BMAX_R; r++)
                if (r < R0) Ys[i1 + I1 * (r + R0 * r2)] = acc[r];
        }
        gsync(g);
        ggram(Ys, I1, R0 * R2, Ss, g);
        gsubspace(Ss, I1, U1, R1, a.inner, Zs, Gs, bad, g);
        // Mode 3 from X: T2 = X x_1 U0^T (R0 x I1 x I2), then Y_(3).
        const int R0I1 = R0 * I1;
        for (int q = g.lt; q < I1 * I2; q += g.gs) {
            const int64_t base = (int64_t)I0 * q;
            double acc[BMAX_R] = {};
#pragma unroll 4
            for (int i0 = 0; i0 < I0; i0++) {
                const double x = X[base + i0];
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R0) acc[r] = fma(x, U0[i0 + I0 * r], acc[r]);
            }
#pragma unroll
            for (int r = 0; r < BMAX_R; r++)
                if (r < R0) T[r + R0 * q] = acc[r];
        }
        gsync(g);
        // Y_(3)[i2, r0 + R0 r1] = sum_i1 T2[r0, i1, i2] U1[i1, r1]
        for (int q = g.lt; q < R0 * I2; q += g.gs) {
            const int r0 = q % R0, i2 = q / R0;
            double acc[BMAX_R] = {};
#pragma unroll 4
            for (int i1 = 0; i1 < I1; i1++) {
                const double v = T[r0 + R0 * i1 + R0I1 * i2];
#pragma unroll
                for (int r = 0; r < BMAX_R; r++)
                    if (r < R1) acc[r] = fma(v, U1[i1 + I1 * r], acc[r]);
            }
#pragma unroll
            for (int r = 0; r < BMAX_R; r++)
                if (r < R1) Ys[i2 + I2 * (r0 + R0 * r)] = acc[r];
        }
        gsync(g);
        ggram(Ys, I2, R0 * R1, Ss, g);
        gsubspace(Ss, I2, U2, R2, a.inner, Zs, Gs, bad, g);
    }
    // Core G[k + K r2] = sum_i2 Y_(3)[i2, k] U2[i2, r2] (the last Y_(3) and U2
    // are those of the final sweep), relative error in FP64.
    const int K = R0 * R1;
    double *Gout = a.G + a.goff[t];
    double g2 = 0.0;
    for (int e = g.lt; e < K * R2; e += g.gs) {
        const int k = e % K, r2 = e / K;
        double acc = 0.0;
        for (int i2 = 0; i2 < I2; i2++) acc = fma(Ys[i2 + I2 * k], U2[i2 + I2 * r2], acc);
        Gout[e] = acc;
        g2 = fma(acc, acc, g2);
    }
    g2 = gsum(g2, red, g);
    // A non-finite input gives a NaN error (fmax would turn NaN into 0).
    const double q = 1.0 - g2 / x2;
    if (g.lt == 0) a.relerr[t] = isnan(q) ? q : sqrt(fmax(0.0, q));
    for (int e = g.lt; e < I0 * R0; e += g.gs) ug[0][e] = U0[e];
    for (int e = g.lt; e < I1 * R1; e += g.gs) ug[1][e] = U1[e];
    for (int e = g.lt; e < I2 * R2; e += g.gs) ug[2][e] = U2[e];
}

template <int NT>
__global__ void __launch_bounds__(NT, (NT <= 256 ? 2 : 1)) batched_hooi_kernel(const BatchArgs *__restrict__ ap) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int cur;
    __shared__ int bad[4];
    const BatchArgs a = *ap;
    double *scr = a.scratch + (int64_t)blockIdx.x * SCR;
    for (;;) {
        if (threadIdx.x == 0) cur = atomicAdd(a.queue, 1);
        __syncthreads();
        const int it = cur;
        __syncthreads();
        if (it >= a.nitems) break;
        const Item item = a.items[it];
        const int gsz = NT / item.g;
        const int gid = threadIdx.x / gsz;
        const Grp g{(int)threadIdx.x % gsz, gsz, 1 + gid};
        const int t = item.t[gid];
        if (t >= 0)
            hooi_one(a, t, sm + (SLOT / item.g) * gid, scr + (SCR / item.g) * gid, g, &bad[gid]);
        __syncthreads();
    }
}

size_t batched_smem() { return (size_t)SLOT * sizeof(double); }

template <int NT>
void kernel_attrs(dt_ctx *ctx, int *per_sm) {
    smem_limit(ctx, batched_hooi_kernel<NT>, batched_smem());
    DT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batched_hooi_kernel<NT>, NT,
                                                          batched_smem()));
}

// Resident CTAs per SM x SMs for a block size.
unsigned batched_grid(dt_ctx *ctx, int nt) {
    int per_sm = 1;
    if (nt == 128)
        kernel_attrs<128>(ctx, &per_sm);
    else if (nt == 512)
        kernel_attrs<512>(ctx, &per_sm);
    else
        kernel_attrs<256>(ctx, &per_sm);
    return (unsigned)(std::max(1, per_sm) * ctx->num_sms);
}

void enqueue_kernel(dt_ctx *ctx, int nt, unsigned grid, const BatchArgs *dargs, int *queue) {
    DT_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), ctx->stream));
    const size_t smem = batched_smem();
    if (nt == 128)
        DT_LAUNCH(ctx, batched_hooi_kernel<128>, grid, 128, smem, dargs);
    else if (nt == 512)
        DT_LAUNCH(ctx, batched_hooi_kernel<512>, grid, 512, smem, dargs);
    else
        DT_LAUNCH(ctx, batched_hooi_kernel<256>, grid, 256, smem, dargs);
}

// Estimated cost of one tensor's sweep (FP64 FMAs): the two passes over X, the
// small contractions, the Grams and the subspace steps.
double tensor_cost(const int64_t *I, const int64_t *R, int inner) {
    const double x = (double)I[0] * I[1] * I[2];
    double c = x * (R[2] + R[0]);
    c += (double)I[0] * I[1] * R[2] * (R[1] + R[0]) + (double)R[0] * I[1] * I[2] * R[1];
    for (int n = 0; n < 3; n++) {
        const double K = (double)R[(n + 1) % 3] * R[(n + 2) % 3];
        c += (double)I[n] * I[n] * K * 0.5 + inner * (double)I[n] * I[n] * R[n] * 2.0;
    }
    return c;
}

// Packs tensors (sorted by cost, descending) into items.  pack >= 1 pairs
// tensors with largest mode <= PAIR_MAX_I, pack >= 2 puts those with largest
// mode <= QUAD_MAX_I four to an item.  Items come out cost-descending.
std::vector<Item> make_items(const std::vector<int> &order, const std::vector<double> &cost,
                             const std::vector<int> &maxI, int pack) {
    std::vector<std::pair<double, Item>> v;
    std::vector<int> pairs, quads;
    for (int t : order) {
        if (pack >= 2 && maxI[t] <= QUAD_MAX_I)
            quads.push_back(t);
        else if (pack >= 1 && maxI[t] <= PAIR_MAX_I)
            pairs.push_back(t);
        else
            v.push_back({cost[t], Item{1, {t, -1, -1, -1}}});
    }
    auto group = [&](const std::vector<int> &ts, int g) {
        for (size_t i = 0; i < ts.size(); i += g) {
            Item it{g, {-1, -1, -1, -1}};
            double c = 0.0;
            for (int k = 0; k < g && i + k < ts.size(); k++) {
                it.t[k] = ts[i + k];
                c = std::max(c, cost[ts[i + k]]);
            }
            // A group of g shares the CTA: it runs about as long as its most
            // expensive member with g times fewer threads.
            v.push_back({c * g, it});
        }
    };
    group(pairs, 2);
    group(quads, 4);
    std::stable_sort(v.begin(), v.end(),
                     [](const std::pair<double, Item> &a, const std::pair<double, Item> &b) {
                         return a.first > b.first;
                     });
    std::vector<Item> out;
    out.reserve(v.size());
    for (auto &p : v) out.push_back(p.second);
    return out;
}

}  // namespace

// Per-context state: tuned configurations per batch signature, the
// instantiated graphs per launch shape, and the device buffers they read.
struct BatchedState {
    std::map<std::vector<int64_t>, std::pair<int, int>> tuned;  // -> (threads, pack)
    std::map<std::pair<int, unsigned>, cudaGraphExec_t> graphs;  // (threads, grid)
    DevMem args, queue, scratch, tables;
    size_t tables_bytes = 0;
    unsigned scratch_grid = 0;
    ~BatchedState() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    }
};

}  // namespace dt

using namespace dt;

extern "C" {

int dt_hooi_batched(dt_ctx *ctx, int count, const int64_t *shapes, const int64_t *ranks,
                    const float *X, const int64_t *x_offsets, int sweeps, int inner_iters,
                    double *U, const int64_t *u_offsets, double *G, const int64_t *g_offsets,
                    double *relerr, int block_threads, dt_batched_report *report) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(count >= 1 && shapes && ranks && X && x_offsets && U && u_offsets && G &&
                         g_offsets && relerr,
                     "dt_hooi_batched: bad arguments");
        DT_CHECK_ARG(sweeps >= 1 && inner_iters >= 1, "dt_hooi_batched: sweeps/inner must be >= 1");
        DT_CHECK_ARG(block_threads == 0 || block_threads == 128 || block_threads == 256 ||
                         block_threads == 512,
                     "dt_hooi_batched: block_threads must be 0 (autotune), 128, 256 or 512");
        int64_t xn = 0, un = 0, gn = 0;
        int64_t maxI = 0, maxR = 0;
        std::vector<double> cost(count);
        std::vector<int> tmaxI(count);
        int n_pair = 0, n_quad = 0;
        for (int t = 0; t < count; t++) {
            int64_t xs = 1, gs = 1, mi = 0;
            for (int m = 0; m < 3; m++) {
                const int64_t I = shapes[3 * t + m], R = ranks[3 * t + m];
                DT_CHECK_ARG(I >= 1 && I <= BMAX_I && R >= 1 && R <= BMAX_R && R <= I,
                             "dt_hooi_batched: tensor %d mode %d: need 1 <= R <= I, I <= %d, R <= %d",
                             t, m, BMAX_I, BMAX_R);
                DT_CHECK_ARG(u_offsets[3 * t + m] >= 0, "dt_hooi_batched: negative U offset");
                xs *= I;
                gs *= R;
                un = std::max(un, u_offsets[3 * t + m] + I * R);
                mi = std::max(mi, I);
                maxR = std::max(maxR, R);
            }
            DT_CHECK_ARG(x_offsets[t] >= 0 && g_offsets[t] >= 0,
                         "dt_hooi_batched: negative X or G offset");
            maxI = std::max(maxI, mi);
            tmaxI[t] = (int)mi;
            n_pair += mi <= PAIR_MAX_I;
            n_quad += mi <= QUAD_MAX_I;
            cost[t] = tensor_cost(shapes + 3 * t, ranks + 3 * t, inner_iters);
            xn = std::max(xn, x_offsets[t] + xs);
            gn = std::max(gn, g_offsets[t] + gs);
        }
        std::vector<int> order(count);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return cost[a] > cost[b]; });
        const std::vector<int64_t> sig = {count, maxI, maxR, sweeps, inner_iters, n_pair, n_quad};
        DT_CUDA(cudaSetDevice(ctx->device));
        if (!ctx->batched) ctx->batched = std::make_shared<BatchedState>();
        BatchedState &st = *std::static_pointer_cast<BatchedState>(ctx->batched);
        DevView xv(ctx, X, xn * sizeof(float), true, false);
        DevView uv(ctx, U, un * sizeof(double), true, true);
        DevView gv(ctx, G, gn * sizeof(double), false, true);
        DevView ev(ctx, relerr, count * sizeof(double), false, true);
        if (!st.args.get()) {
            st.args.alloc(ctx, sizeof(BatchArgs));
            st.queue.alloc(ctx, sizeof(int));
        }
        const int64_t launches0 = ctx->launches;

        // Descriptor tables (shapes, ranks, offsets, items) in one device
        // buffer kept on the context; `items` is rebuilt per configuration.
        auto upload = [&](const std::vector<Item> &items, BatchArgs &a) {
            const size_t n3 = 3 * (size_t)count;
            const size_t bytes = (3 * n3 + 2 * (size_t)count) * sizeof(int64_t) +
                                 items.size() * sizeof(Item);
            std::vector<char> h(bytes);
            int64_t *p = reinterpret_cast<int64_t *>(h.data());
            std::memcpy(p, shapes, n3 * sizeof(int64_t));
            std::memcpy(p + n3, ranks, n3 * sizeof(int64_t));
            std::memcpy(p + 2 * n3, u_offsets, n3 * sizeof(int64_t));
            std::memcpy(p + 3 * n3, x_offsets, count * sizeof(int64_t));
            std::memcpy(p + 3 * n3 + count, g_offsets, count * sizeof(int64_t));
            std::memcpy(p + 3 * n3 + 2 * count, items.data(), items.size() * sizeof(Item));
            if (st.tables_bytes < bytes) {
                st.tables.alloc(ctx, bytes);
                st.tables_bytes = bytes;
            }
            DT_CUDA(cudaMemcpyAsync(st.tables.get(), h.data(), bytes, cudaMemcpyHostToDevice,
                                    ctx->stream));
            const int64_t *d = st.tables.as<int64_t>();
            a.count = count;
            a.nitems = (int)items.size();
            a.shape = d;
            a.rank = d + n3;
            a.uoff = d + 2 * n3;
            a.xoff = d + 3 * n3;
            a.goff = d + 3 * n3 + count;
            a.items = reinterpret_cast<const Item *>(d + 3 * n3 + 2 * count);
            // The host copy must outlive the asynchronous copy from pageable
            // memory only until the call returns; the runtime stages it.
            DT_CUDA(cudaStreamSynchronize(ctx->stream));
        };
        auto ensure_scratch = [&](unsigned grid) {
            if (st.scratch_grid < grid) {
                st.scratch.alloc(ctx, (size_t)grid * SCR * sizeof(double));
                st.scratch_grid = grid;
            }
        };
        BatchArgs base{};
        base.X = xv.as<float>();
        base.G = gv.as<double>();
        base.relerr = ev.as<double>();
        base.sweeps = sweeps;
        base.inner = inner_iters;
        base.queue = st.queue.as<int>();

        int nt = block_threads, pack = 0;
        int timed = 0;
        double tune_best = 0.0, tune_worst = 0.0;
        if (nt != 0) {
            pack = 2;  // pairs and quads where they fit; no autotuning
        } else {
            auto itc = st.tuned.find(sig);
            if (itc != st.tuned.end()) {
                nt = itc->second.first;
                pack = itc->second.second;
            } else {
                // Autotune on a stratified sample (every k-th tensor of the
                // cost order) with a scratch copy of U.  The sample must fill
                // the largest grid several times over, or configurations with
                // few large CTAs win on the sample and lose on the batch: up
                // to 8192 tensors, the whole batch is timed.
                const int sample = std::min(count, 8192);
                std::vector<int> sord;
                for (int i = 0; i < sample; i++)
                    sord.push_back(order[(int64_t)i * count / sample]);
                DevMem ucopy(ctx, un * sizeof(double));
                float best = 1e30f, worst = 0.f;
                const int cand_nt[3] = {128, 256, 512};
                for (int c = 0; c < 3; c++) {
                    for (int pk = 0; pk <= 2; pk++) {
                        if (pk == 1 && n_pair == 0) continue;
                        if (pk == 2 && n_quad == 0) continue;
                        BatchArgs b = base;
                        upload(make_items(sord, cost, tmaxI, pk), b);
                        b.U = ucopy.as<double>();
                        const unsigned grid = batched_grid(ctx, cand_nt[c]);
                        ensure_scratch(grid);
                        b.scratch = st.scratch.as<double>();
                        DT_CUDA(cudaMemcpyAsync(st.args.get(), &b, sizeof(b),
                                                cudaMemcpyHostToDevice, ctx->stream));
                        float ms = 0.f;
                        for (int rep = 0; rep < 2; rep++) {  // warm, then timed
                            DT_CUDA(cudaMemcpyAsync(ucopy.get(), uv.ptr(), un * sizeof(double),
                                                    cudaMemcpyDeviceToDevice, ctx->stream));
                            DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
                            enqueue_kernel(ctx, cand_nt[c], grid, st.args.as<BatchArgs>(),
                                           st.queue.as<int>());
                            DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
                            DT_CUDA(cudaEventSynchronize(ctx->ev_stop));
                            DT_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
                        }
                        timed++;
                        worst = std::max(worst, ms);
                        if (ms < best) {
                            best = ms;
                            nt = cand_nt[c];
                            pack = pk;
                        }
                    }
                }
                tune_best = best;
                tune_worst = worst;
                st.tuned[sig] = {nt, pack};
            }
        }
        const unsigned grid = batched_grid(ctx, nt);
        ensure_scratch(grid);
        const std::vector<Item> items = make_items(order, cost, tmaxI, pack);
        BatchArgs a = base;
        upload(items, a);
        a.U = uv.as<double>();
        a.scratch = st.scratch.as<double>();
        DT_CUDA(cudaMemcpyAsync(st.args.get(), &a, sizeof(a), cudaMemcpyHostToDevice,
                                ctx->stream));
        // The graph (queue reset + persistent kernel) for this launch shape:
        // captured once, replayed by every later call.
        const std::pair<int, unsigned> gkey(nt, grid);
        int reused = 1;
        // Streams that cannot be captured (the legacy and per-thread default
        // streams) run the launch directly.
        const bool capturable = ctx->stream != nullptr && ctx->stream != cudaStreamLegacy &&
                                ctx->stream != cudaStreamPerThread;
        if (!capturable) {
            DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
            enqueue_kernel(ctx, nt, grid, st.args.as<BatchArgs>(), st.queue.as<int>());
            DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
            reused = 0;
        }
        auto itg = capturable ? st.graphs.find(gkey) : st.graphs.end();
        if (capturable && itg == st.graphs.end()) {
            reused = 0;
            cudaGraph_t graph;
            cudaGraphExec_t exec;
            DT_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            const int64_t l0 = ctx->launches;
            try {
                enqueue_kernel(ctx, nt, grid, st.args.as<BatchArgs>(), st.queue.as<int>());
            } catch (...) {
                cudaStreamEndCapture(ctx->stream, &graph);
                throw;
            }
            ctx->launches = l0;  // counted when the graph is launched
            DT_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            DT_CUDA(ie);
            itg = st.graphs.emplace(gkey, exec).first;
        }
        if (capturable) {
            DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
            DT_CUDA(cudaGraphLaunch(itg->second, ctx->stream));
            ctx->launches++;
            DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
        }
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        float ms = 0.f;
        DT_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        uv.finish();
        gv.finish();
        ev.finish();
        if (report) {
            std::memset(report, 0, sizeof(*report));
            report->device_ms = ms;
            report->block_threads = nt;
            report->grid = (int)grid;
            report->kernel_launches = (int)(ctx->launches - launches0);
            report->pack = pack;
            report->items = (int)items.size();
            report->candidates_timed = timed;
            report->tune_best_ms = tune_best;
            report->tune_worst_ms = tune_worst;
            report->graph_reused = reused;
        }
    });
}

}  // extern "C"
