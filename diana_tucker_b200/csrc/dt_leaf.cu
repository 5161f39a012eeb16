// The leaf Gram of the mixed-precision dense HOOI, without forming Y_(n).
//
// In the dimension tree a pair node {p, q = p + 1} holds T, the input
// contracted in every mode but p and q (modes p and q keep I_p, I_q, every
// other mode has extent R).  Leaf p needs
//     S_p = Y_(p) Y_(p)^T,   Y_(p) = (T x_q U_q^T)_(p),
// and, over the slices T_c (I_p x I_q, c running over the other modes),
//     S_p = sum_c W_c W_c^T,   W_c = T_c U_q   (I_p x R_q),
// (leaf q is the same with T_c^T and the new U_p).  One launch reads T once:
// each CTA takes a run of consecutive slices, forms W_c in FP32 from the
// split BF16 T (hi + lo) and FP32 U, and adds W_c W_c^T into an FP64 block of
// S_p held in registers (a 6 x 6, 4 x 4 or 2 x 2 block per thread); the
// per-CTA partials are then summed in a fixed order by a second kernel.  This
// replaces the leaf contraction (writing Y_(p), 1.5 MB for 96 x 4096 split
// BF16), its Gram and the Gram's split-K partials with two light launches.
//
// The sweep core's norm needs no core either: ||G||^2 = ||U_n^T Y_(n)||^2 =
// trace(U_n^T S_n U_n) for the last mode (quad_trace_kernel).
#include <cuda_bf16.h>

#include <algorithm>

#include "dt_kernels.cuh"
#include "dt_leaf.cuh"

namespace dt {
namespace {

constexpr int SG_THREADS = 256;

// Slices [c0, c0 + cg) of T: element (i, j, c) (i < np along mode p, j < nq
// along mode q) at i * sp + j * sq + (c % clo) + (c / clo) * chs.
struct SliceView {
    const __nv_bfloat16 *hi, *lo;
    int np, nq;
    int64_t sp, sq;
    int64_t clo, chs;
    int nc;
};

constexpr int SG_MAXCG = 64;  // slices per CTA at most

template <int BS>
__global__ void __launch_bounds__(SG_THREADS, 2) slice_gram_kernel(SliceView v, int side, int cg,
                                                                 const double *__restrict__ U,
                                                                 int R, double *__restrict__ part) {
    // side 0: S over mode p, W = T_c U_q (contract mode q); side 1: the reverse.
    extern __shared__ float sgm[];
    __shared__ int64_t coff[SG_MAXCG];
    const int na = side == 0 ? v.np : v.nq;  // S dimension
    const int nb = side == 0 ? v.nq : v.np;  // contracted dimension
    const int pitch = v.np + 1;              // slice stored [j][i] with padded rows
    const int RP = (R + 3) & ~3;
    const int WP = RP + 1;                   // odd pitch: the S-phase loads spread over banks
    float *Zs = sgm;                              // cg x nq x pitch
    float *Us = Zs + (size_t)cg * v.nq * pitch;   // nb x RP
    float *Ws = Us + (size_t)nb * RP;             // na x WP (row a at a * WP)
    const int c0 = blockIdx.x * cg;
    const int ncg = min(cg, v.nc - c0);
    pdl_trigger();
    if (threadIdx.x < ncg) {
        const int64_t c = c0 + threadIdx.x;
        coff[threadIdx.x] = (c % v.clo) + (c / v.clo) * v.chs;
    }
    pdl_wait();
    for (int e = threadIdx.x; e < nb * RP; e += SG_THREADS) {
        const int b = e / RP, r = e - b * RP;
        Us[e] = r < R ? (float)U[b + (int64_t)nb * r] : 0.f;
    }
    __syncthreads();
    // Load the CTA's slices.  The element index runs over three digits (the
    // contiguous one fastest: c when the low part of c is contiguous in T,
    // clo > 1; else i); each thread steps by SG_THREADS with carries, so the
    // loop divides nothing.
    {
        const bool c_inner = v.clo > 1;
        const int n0 = c_inner ? ncg : v.np, n1 = c_inner ? v.np : v.nq;
        const int total = ncg * v.np * v.nq;
        const int k0 = SG_THREADS % n0, k1 = (SG_THREADS / n0) % n1,
                  k2 = SG_THREADS / (n0 * n1);
        int d0 = threadIdx.x % n0, d1 = (threadIdx.x / n0) % n1, d2 = threadIdx.x / (n0 * n1);
        constexpr int UNR = 4;  // elements per thread and round: 2 UNR loads in flight
        for (int e = threadIdx.x; e < total; e += UNR * SG_THREADS) {
            int64_t off[UNR];
            int dst[UNR];
#pragma unroll
            for (int u = 0; u < UNR; u++) {
                const int cc = c_inner ? d0 : d2, i = c_inner ? d1 : d0, j = c_inner ? d2 : d1;
                const bool on = e + u * SG_THREADS < total;
                off[u] = on ? i * v.sp + j * v.sq + coff[cc] : 0;
                dst[u] = on ? (cc * v.nq + j) * pitch + i : -1;
                d0 += k0;
                d1 += k1;
                d2 += k2;
                if (d0 >= n0) {
                    d0 -= n0;
                    d1++;
                }
                if (d1 >= n1) {
                    d1 -= n1;
                    d2++;
                }
            }
            float hv[UNR], lv[UNR];
#pragma unroll
            for (int u = 0; u < UNR; u++) {
                hv[u] = dst[u] >= 0 ? __bfloat162float(v.hi[off[u]]) : 0.f;
                lv[u] = dst[u] >= 0 && v.lo ? __bfloat162float(v.lo[off[u]]) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < UNR; u++)
                if (dst[u] >= 0) Zs[dst[u]] = hv[u] + lv[u];
        }
    }
    __syncthreads();
    // This thread's BS x BS block of S: rows bi*BS.., columns bj*BS.. of the
    // 16 x 16 grid of blocks.
    const int bi = threadIdx.x & 15, bj = threadIdx.x >> 4;
    double acc[BS][BS];
#pragma unroll
    for (int x = 0; x < BS; x++)
#pragma unroll
        for (int y = 0; y < BS; y++) acc[x][y] = 0.0;
    for (int cc = 0; cc < ncg; cc++) {
        const float *Z = Zs + (size_t)cc * v.nq * pitch;
        // W[a][r] = sum_b Z(a, b) U[b][r]; Z(a, b) = Z[b][a] (side 0) or Z[a][b].
        for (int o = threadIdx.x; o < na * RP; o += SG_THREADS) {
            const int a = o % na, r = o / na;
            float s0 = 0.f, s1 = 0.f;
            int b = 0;
            if (side == 0) {
                for (; b + 1 < nb; b += 2) {
                    s0 = fmaf(Z[b * pitch + a], Us[b * RP + r], s0);
                    s1 = fmaf(Z[(b + 1) * pitch + a], Us[(b + 1) * RP + r], s1);
                }
                if (b < nb) s0 = fmaf(Z[b * pitch + a], Us[b * RP + r], s0);
            } else {
                for (; b + 1 < nb; b += 2) {
                    s0 = fmaf(Z[a * pitch + b], Us[b * RP + r], s0);
                    s1 = fmaf(Z[a * pitch + b + 1], Us[(b + 1) * RP + r], s1);
                }
                if (b < nb) s0 = fmaf(Z[a * pitch + b], Us[b * RP + r], s0);
            }
            Ws[a * WP + r] = s0 + s1;
        }
        __syncthreads();
        for (int r = 0; r < R; r++) {
            double wa[BS], wb[BS];
#pragma unroll
            for (int x = 0; x < BS; x++) {
                const int ia = bi * BS + x, ib = bj * BS + x;
                wa[x] = ia < na ? (double)Ws[ia * WP + r] : 0.0;
                wb[x] = ib < na ? (double)Ws[ib * WP + r] : 0.0;
            }
#pragma unroll
            for (int x = 0; x < BS; x++)
#pragma unroll
                for (int y = 0; y < BS; y++) acc[x][y] = fma(wa[x], wb[y], acc[x][y]);
        }
        __syncthreads();
    }
    double *dst = part + (int64_t)blockIdx.x * na * na;
#pragma unroll
    for (int x = 0; x < BS; x++)
#pragma unroll
        for (int y = 0; y < BS; y++) {
            const int i = bi * BS + x, j = bj * BS + y;
            if (i < na && j < na) dst[i + (int64_t)na * j] = acc[x][y];
        }
}

// S[e] = sum_z part[z][e], z in order.
__global__ void sum_parts_fixed_kernel(const double *__restrict__ part, int nz, int64_t n,
                                       double *__restrict__ S) {
    pdl_trigger();
    pdl_wait();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        // Eight loads in flight, added in z order.
        double s = 0.0;
        int z = 0;
        for (; z + 8 <= nz; z += 8) {
            double v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] = part[(int64_t)(z + q) * n + e];
#pragma unroll
            for (int q = 0; q < 8; q++) s += v[q];
        }
        for (; z < nz; z++) s += part[(int64_t)z * n + e];
        S[e] = s;
    }
}

// out = sum_r U(:, r)^T S U(:, r) for S n x n, U n x R (col-major), FP64.
__global__ void __launch_bounds__(256) quad_trace_kernel(const double *__restrict__ S, int n,
                                                         const double *__restrict__ U, int R,
                                                         double *__restrict__ out) {
    pdl_trigger();
    pdl_wait();
    double s = 0.0;
    for (int o = threadIdx.x; o < n * R; o += blockDim.x) {
        const int i = o % n, r = o / n;
        const double *u = U + (int64_t)n * r;
        double t0 = 0.0, t1 = 0.0;
        int j = 0;
        for (; j + 1 < n; j += 2) {
            t0 = fma(S[i + (int64_t)n * j], u[j], t0);
            t1 = fma(S[i + (int64_t)n * (j + 1)], u[j + 1], t1);
        }
        if (j < n) t0 = fma(S[i + (int64_t)n * j], u[j], t0);
        s = fma(u[i], t0 + t1, s);
    }
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        *out = t;
    }
}

// ---------------------------------------------------------------------------
// Leading-R subspace of a small symmetric S (n <= 128) in one CTA, FP64:
// L <- orth(S^iters L) with CholeskyQR after every second product and a
// second CholeskyQR pass at the end (CholeskyQR2), on the FP64 tensor cores.
//
//  * S, L and Z live in shared memory, column-major with pitches = 4 mod 16
//    doubles, so the m8n8k4 fragment loads (rows g + 8 m, k t + 4 s) hit 16
//    distinct bank pairs per half warp; rows beyond n and columns beyond R
//    are zero.
//  * Products Z = S L: warp w takes output tiles w, w + 8, ... (8 x 8 each)
//    and runs their k-loop; the R x R Gram Z^T Z likewise (no cross-warp
//    reduction).
//  * Cholesky of the Gram by one warp (lane j holds column j), then the rows
//    of Q = Z R^-1 by forward substitution, one thread per row, the updates
//    of the later columns independent of each other.
//  * A non-positive pivot (a rank-deficient product) falls back to modified
//    Gram-Schmidt by one warp and sets bit 2 of *flag.
//  * With g2_out, the final trace(Q^T S Q) (the norm^2 of the core of the
//    last mode, used for the sweep residual) is written there.
// ---------------------------------------------------------------------------
// A pure function of its operands (no volatile): the compiler may hoist the
// shared-memory loads of later k-steps ahead of earlier MMAs.
__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

__host__ __device__ constexpr int pitch4(int n) { return n + ((4 - n % 16) + 16) % 16; }

constexpr int SS_THREADS = 256;
constexpr int SS_MAXT = 8;  // output tiles per warp of one product (npad <= 128, RM <= 32)

// Z (npad x RM, pitch pz) = S (npad x npad, pitch ps) A (npad x RM, pitch pa).
// Warp w owns tiles w, w + 8, ...; their k-loops run interleaved (independent
// accumulators), so the MMA latency overlaps across tiles.
template <int RM>
__device__ void ss_product(const double *S, int ps, const double *A, int pa, double *Z, int pz,
                           int npad) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mt_n = npad / 8, tiles = mt_n * (RM / 8);
    const double *sa[SS_MAXT], *sb[SS_MAXT];
    double d0[SS_MAXT], d1[SS_MAXT];
    int nt = 0;
#pragma unroll
    for (int q = 0; q < SS_MAXT; q++) {
        const int tile = w + 8 * q;
        const bool on = tile < tiles;
        const int mt = on ? tile % mt_n : 0, ntl = on ? tile / mt_n : 0;
        sa[q] = S + 8 * mt + g + (int64_t)ps * t;
        sb[q] = A + t + (int64_t)pa * (8 * ntl + g);
        d0[q] = d1[q] = 0.0;
        nt += on;
    }
    for (int k = 0; k < npad; k += 4) {
#pragma unroll
        for (int q = 0; q < SS_MAXT; q++)
            if (q < nt) dmma884(d0[q], d1[q], sa[q][(int64_t)ps * k], sb[q][k]);
    }
#pragma unroll
    for (int q = 0; q < SS_MAXT; q++) {
        if (q >= nt) break;
        const int tile = w + 8 * q, mt = tile % mt_n, ntl = tile / mt_n;
        Z[8 * mt + g + (int64_t)pz * (8 * ntl + 2 * t)] = d0[q];
        Z[8 * mt + g + (int64_t)pz * (8 * ntl + 2 * t + 1)] = d1[q];
    }
}

// Q (in place over Z, pitch pz) = orth(Z) by one CholeskyQR pass; Gs is RM x
// RM scratch.  Returns false (nothing changed) on a non-positive pivot.
template <int RM>
__device__ bool ss_cholqr(double *Z, int pz, int n, int npad, int R, double *Gs, int *bad) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    constexpr int NT = RM / 8;
    double *Dinv = Gs + RM * RM;  // 1 / R(k, k)
    for (int tile = w; tile < NT * NT; tile += SS_THREADS / 32) {
        const int ma = tile % NT, mb = tile / NT;
        // Two accumulator pairs (even / odd k-steps), added at the end.
        double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
        const double *za = Z + t + (int64_t)pz * (8 * ma + g);
        const double *zb = Z + t + (int64_t)pz * (8 * mb + g);
        int k = 0;
        for (; k + 8 <= npad; k += 8) {
            dmma884(d0, d1, za[k], zb[k]);
            dmma884(e0, e1, za[k + 4], zb[k + 4]);
        }
        for (; k < npad; k += 4) dmma884(d0, d1, za[k], zb[k]);
        Gs[(8 * ma + g) * RM + 8 * mb + 2 * t] = d0 + e0;
        Gs[(8 * ma + g) * RM + 8 * mb + 2 * t + 1] = d1 + e1;
    }
    __syncthreads();
    if (w == 0) {
        // Lane j holds column j of the Gram; on exit column j of R (upper).
        // One reciprocal square root per pivot, no division.
        double c[RM];
#pragma unroll
        for (int i = 0; i < RM; i++) c[i] = (lane < R && i < R) ? Gs[i * RM + lane] : 0.0;
        const double g00 = __shfl_sync(0xffffffffu, c[0], 0);
        bool ok = true;
#pragma unroll
        for (int k = 0; k < RM; k++) {
            if (k >= R) break;
            const double dkk = __shfl_sync(0xffffffffu, c[k], k);
            if (!(dkk > 1e-28 * g00)) ok = false;
            const double inv = rsqrt(fmax(dkk, 1e-300));
            if (lane == k) Dinv[k] = inv;
            c[k] = lane == k ? dkk * inv : (lane > k ? c[k] * inv : c[k]);
#pragma unroll
            for (int i = k + 1; i < RM; i++) {
                if (i >= R) break;
                const double rki = __shfl_sync(0xffffffffu, c[k], i);
                if (lane >= i) c[i] = fma(-rki, c[k], c[i]);
            }
        }
        if (lane < R) {
#pragma unroll
            for (int i = 0; i < RM; i++)
                if (i < R) Gs[i * RM + lane] = i <= lane ? c[i] : 0.0;
        }
        if (lane == 0) *bad = ok ? 0 : 1;
    }
    __syncthreads();
    if (*bad) return false;
    // Row i: q_c = (z_c - sum_{k<c} q_k R(k, c)) / R(c, c); the updates of the
    // later columns are independent of each other.
    for (int i = threadIdx.x; i < n; i += SS_THREADS) {
        double z[RM];
#pragma unroll
        for (int c = 0; c < RM; c++) z[c] = c < R ? Z[i + (int64_t)pz * c] : 0.0;
#pragma unroll
        for (int k = 0; k < RM; k++) {
            if (k >= R) break;
            const double q = z[k] * Dinv[k];
            z[k] = q;
#pragma unroll
            for (int c = k + 1; c < RM; c++)
                if (c < R) z[c] = fma(-q, Gs[k * RM + c], z[c]);
        }
#pragma unroll
        for (int c = 0; c < RM; c++)
            if (c < R) Z[i + (int64_t)pz * c] = z[c];
    }
    __syncthreads();
    (void)npad;
    return true;
}

// Modified Gram-Schmidt over the R columns of Z by one warp (zero columns
// stay zero).
__device__ void ss_mgs(double *Z, int pz, int n, int R) {
    if ((threadIdx.x >> 5) == 0) {
        const int lane = threadIdx.x & 31;
        for (int c = 0; c < R; c++) {
            double *zc = Z + (int64_t)pz * c;
            for (int p = 0; p < c; p++) {
                const double *zp = Z + (int64_t)pz * p;
                double d = 0.0;
                for (int i = lane; i < n; i += 32) d = fma(zc[i], zp[i], d);
                for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
                for (int i = lane; i < n; i += 32) zc[i] = fma(-d, zp[i], zc[i]);
                __syncwarp();
            }
            double s = 0.0;
            for (int i = lane; i < n; i += 32) s = fma(zc[i], zc[i], s);
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            const double inv = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
            for (int i = lane; i < n; i += 32) zc[i] *= inv;
            __syncwarp();
        }
    }
    __syncthreads();
}

template <int RM>
__global__ void __launch_bounds__(SS_THREADS) subspace_small_kernel(const double *__restrict__ Sg,
                                                                    int n, double *__restrict__ Lg,
                                                                    int R, int iters,
                                                                    int *__restrict__ flag,
                                                                    double *__restrict__ g2_out) {
    extern __shared__ __align__(16) double ssm[];
    __shared__ int bad;
    const int npad = (n + 7) & ~7;
    const int ps = pitch4(npad), pz = pitch4(npad);
    double *S = ssm;                          // npad columns of pitch ps
    double *A = S + (size_t)ps * npad;        // RM columns of pitch pz
    double *Z = A + (size_t)pz * RM;
    double *Gs = Z + (size_t)pz * RM;         // RM x RM
    pdl_trigger();
    // Zero everything the padding reads.
    for (int e = threadIdx.x; e < (ps * npad + 2 * pz * RM); e += SS_THREADS) ssm[e] = 0.0;
    __syncthreads();
    pdl_wait();
    for (int e = threadIdx.x; e < n * n; e += SS_THREADS) {
        const int i = e % n, j = e / n;
        S[i + (int64_t)ps * j] = Sg[e];
    }
    for (int e = threadIdx.x; e < n * R; e += SS_THREADS) {
        const int i = e % n, c = e / n;
        A[i + (int64_t)pz * c] = Lg[e];
    }
    __syncthreads();
    double *cur = A, *nxt = Z;
    bool fell_back = false;
    for (int it = 0; it < iters; it++) {
        ss_product<RM>(S, ps, cur, pz, nxt, pz, npad);
        __syncthreads();
        double *tmp = cur;
        cur = nxt;
        nxt = tmp;
        // Orthonormalise after every second product and after the last.
        if ((it & 1) || it + 1 == iters) {
            if (!ss_cholqr<RM>(cur, pz, n, npad, R, Gs, &bad)) {
                ss_mgs(cur, pz, n, R);
                fell_back = true;
            }
        }
    }
    // Second pass (CholeskyQR2): orthonormal to rounding.
    if (!ss_cholqr<RM>(cur, pz, n, npad, R, Gs, &bad)) {
        ss_mgs(cur, pz, n, R);
        fell_back = true;
    }
    for (int e = threadIdx.x; e < n * R; e += SS_THREADS) {
        const int i = e % n, c = e / n;
        Lg[e] = cur[i + (int64_t)pz * c];
    }
    if (fell_back && threadIdx.x == 0) atomicOr(flag, 4);
    if (g2_out) {
        // trace(Q^T S Q) = sum of Q .* (S Q).
        ss_product<RM>(S, ps, cur, pz, nxt, pz, npad);
        __syncthreads();
        double s = 0.0;
        for (int e = threadIdx.x; e < n * R; e += SS_THREADS) {
            const int i = e % n, c = e / n;
            s = fma(cur[i + (int64_t)pz * c], nxt[i + (int64_t)pz * c], s);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) Gs[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tsum = 0.0;
            for (int w = 0; w < SS_THREADS / 32; w++) tsum += Gs[w];
            *g2_out = tsum;
        }
    }
}

}  // namespace

bool subspace_small_supported(int64_t n, int64_t R) {
    return n >= 1 && n <= 128 && R >= 1 && R <= 32 && R <= n;
}

void subspace_small(dt_ctx *ctx, const double *S, int64_t n, double *L, int64_t R, int iters,
                    int *flag, double *g2_out) {
    DT_CHECK_ARG(subspace_small_supported(n, R) && iters >= 1, "subspace_small: n=%lld R=%lld",
                 (long long)n, (long long)R);
    const int npad = (int)((n + 7) & ~int64_t(7));
    const int p = pitch4(npad);
    auto go = [&](auto kernel, int RM) {
        const size_t smem =
            ((size_t)p * npad + 2 * (size_t)p * RM + (size_t)RM * RM + RM) * sizeof(double);
        smem_limit(ctx, kernel, smem);
        DT_LAUNCH_PDL(ctx, kernel, 1, SS_THREADS, smem, S, (int)n, L, (int)R, iters, flag, g2_out);
    };
    if (R <= 8)
        go(subspace_small_kernel<8>, 8);
    else if (R <= 16)
        go(subspace_small_kernel<16>, 16);
    else
        go(subspace_small_kernel<32>, 32);
}

bool pair_gram_supported(int64_t np, int64_t nq, int64_t R) {
    return np >= 1 && nq >= 1 && np <= 128 && nq <= 128 && R >= 1 && R <= 32 &&
           (np + 1) * nq * 4 + std::max(np, nq) * 32 * 4 * 2 <= 200 * 1024;
}

size_t pair_gram_scratch_doubles(int64_t np, int64_t nq, int64_t nc) {
    const int64_t n = std::max(np, nq);
    const int64_t nz = std::max<int64_t>(std::min<int64_t>(nc, 256), (nc + SG_MAXCG - 1) / SG_MAXCG);
    return (size_t)nz * n * n;
}

void pair_gram(dt_ctx *ctx, const __nv_bfloat16 *Th, const __nv_bfloat16 *Tl, int64_t np,
               int64_t nq, int64_t sp, int64_t sq, int64_t clo, int64_t chs, int64_t nc, int side,
               const double *U, int64_t R, double *part, size_t part_doubles, double *S) {
    DT_CHECK_ARG(pair_gram_supported(np, nq, R), "pair_gram: unsupported np=%lld nq=%lld R=%lld",
                 (long long)np, (long long)nq, (long long)R);
    SliceView v{Th, Tl, (int)np, (int)nq, sp, sq, clo, chs, (int)nc};
    const int64_t na = side == 0 ? np : nq, nb = side == 0 ? nq : np;
    const int RP = (int)((R + 3) & ~int64_t(3));
    // Slices per CTA: as many CTAs as SMs where the slices allow, the
    // group's slices staged together within ~160 KB of shared memory.
    const size_t slice_bytes = (size_t)nq * (np + 1) * sizeof(float);
    const size_t fixed = ((size_t)nb * RP + (size_t)na * (RP + 1)) * sizeof(float);
    // Slices per CTA: one while the slices fill two CTAs per SM, more only
    // for a long slice list.
    int cg = (int)std::max<int64_t>(1, (nc + 2 * ctx->num_sms - 1) / (2 * ctx->num_sms));
    cg = std::min(cg, SG_MAXCG);
    while (cg > 1 && fixed + cg * slice_bytes > 160 * 1024) cg--;
    int64_t nz = (nc + cg - 1) / cg;
    while ((size_t)nz * na * na > part_doubles && cg < SG_MAXCG) {
        cg++;
        nz = (nc + cg - 1) / cg;
    }
    DT_CHECK_ARG((size_t)nz * na * na <= part_doubles, "pair_gram: scratch too small");
    DT_CHECK_ARG(fixed + cg * slice_bytes <= 220 * 1024, "pair_gram: slices too large");
    const size_t smem = fixed + cg * slice_bytes;
    auto go = [&](auto kernel) {
        smem_limit(ctx, kernel, smem);
        DT_LAUNCH_PDL(ctx, kernel, (unsigned)nz, SG_THREADS, smem, v, side, cg, U, (int)R, part);
    };
    if (na <= 32)
        go(slice_gram_kernel<2>);
    else if (na <= 64)
        go(slice_gram_kernel<4>);
    else if (na <= 96)
        go(slice_gram_kernel<6>);
    else
        go(slice_gram_kernel<8>);
    const int64_t n2 = na * na;
    DT_LAUNCH_PDL(ctx, sum_parts_fixed_kernel,
                  (unsigned)std::max<int64_t>(1, std::min<int64_t>((n2 + 127) / 128, 4 * ctx->num_sms)),
                  128, 0, part, (int)nz, n2, S);
}

void quad_trace(dt_ctx *ctx, const double *S, int64_t n, const double *U, int64_t R, double *out) {
    DT_LAUNCH_PDL(ctx, quad_trace_kernel, 1, 256, 0, S, (int)n, U, (int)R, out);
}

}  // namespace dt
