// Small dense FP64 linear algebra on the GPU: the reference's LAPACK calls
// (src/operator/operator_double.cpp:84-155) and its ALS_ leading-subspace step
// (template/algorithm/tucker/hooi_als.tpp:7-34), kept on the device so a HOOI
// sweep never round-trips to the host.  These matrices are tiny (R x R, I_n x R,
// I_n x I_n): one CTA per problem, latency-bound, so the code minimises block
// barriers rather than flops.
#include <vector>

#include "dt_kernels.cuh"

namespace dt {
namespace {

constexpr int LA_NT = 512;

__device__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (l == 0) red[32] = v;
    }
    __syncthreads();
    return red[32];
}

// Householder QR of the m x n col-major W (in place: R in the upper triangle,
// reflector tails below the diagonal, tau[j]), then Q (m x n) formed by
// applying H_0 ... H_{n-1} to [I; 0] backwards -- the dgeqrf/dorgqr sequence.
// Reflector (dlarfg): beta = -sign(alpha) ||(alpha, x)||, tau = (beta-alpha)/beta,
// v = [1; x/(alpha-beta)]; tau = 0 when x == 0.
__device__ void hqr_device(double *W, int64_t m, int64_t n, double *tau, double *Q,
                           double *red) {
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31, nwarps = blockDim.x >> 5;
    for (int64_t j = 0; j < n; j++) {
        double *col = W + j * m;
        double s = 0.0;
        for (int64_t i = j + 1 + t; i < m; i += blockDim.x) s = fma(col[i], col[i], s);
        const double xnorm2 = block_sum(s, red);
        const double alpha = col[j];
        double tj, scale;
        if (xnorm2 == 0.0) {
            tj = 0.0;
            scale = 0.0;
        } else {
            const double beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
            tj = (beta - alpha) / beta;
            scale = 1.0 / (alpha - beta);
        }
        __syncthreads();
        if (tj != 0.0) {
            for (int64_t i = j + 1 + t; i < m; i += blockDim.x) col[i] *= scale;
        }
        __syncthreads();
        if (t == 0) {
            tau[j] = tj;
            if (tj != 0.0) col[j] = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
        }
        // Apply H_j to the trailing columns, one warp per column.
        if (tj != 0.0) {
            for (int64_t c = j + 1 + warp; c < n; c += nwarps) {
                double *cc = W + c * m;
                const double cj = cc[j];  // read before lane 0 rewrites it
                double w = 0.0;
                for (int64_t i = j + 1 + lane; i < m; i += 32) w = fma(col[i], cc[i], w);
                for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
                w += cj;
                w *= tj;
                if (lane == 0) cc[j] -= w;
                for (int64_t i = j + 1 + lane; i < m; i += 32) cc[i] = fma(-w, col[i], cc[i]);
            }
        }
        __syncthreads();
    }
    if (!Q) return;
    for (int64_t e = t; e < m * n; e += blockDim.x) {
        const int64_t i = e % m, c = e / m;
        Q[e] = (i == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int64_t j = n - 1; j >= 0; j--) {
        const double tj = tau[j];
        if (tj != 0.0) {
            const double *v = W + j * m;
            for (int64_t c = j + warp; c < n; c += nwarps) {
                double *qc = Q + c * m;
                const double qj = qc[j];  // read before lane 0 rewrites it
                double w = 0.0;
                for (int64_t i = j + 1 + lane; i < m; i += 32) w = fma(v[i], qc[i], w);
                for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
                w += qj;
                w *= tj;
                if (lane == 0) qc[j] -= w;
                for (int64_t i = j + 1 + lane; i < m; i += 32) qc[i] = fma(-w, v[i], qc[i]);
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(LA_NT) hqr_kernel(const double *A, int64_t m, int64_t n,
                                                    double *Q, double *R, double *work) {
    __shared__ double red[33];
    double *W = work;
    double *tau = work + m * n;
    for (int64_t e = threadIdx.x; e < m * n; e += blockDim.x) W[e] = A[e];
    __syncthreads();
    hqr_device(W, m, n, tau, Q, red);
    if (R) {
        for (int64_t e = threadIdx.x; e < n * n; e += blockDim.x) {
            const int64_t i = e % n, c = e / n;
            R[e] = (i <= c) ? W[i + c * m] : 0.0;
        }
    }
}

// Cholesky G = R^T R of the r x r SPD matrix in smem (row-major G[i*r+c]) by
// one warp, then Rinv = R^{-1} (upper, row-major).  Lane c keeps column c in
// registers and rows are exchanged with shuffles, so the r pivots form one
// short dependency chain (one sqrt and one reciprocal per pivot).  Returns
// false on a non-positive pivot.  Runs in warp 0 only; r <= 32.
template <int RMAX, bool INV = true>
__device__ bool warp_chol_inv(double *G, double *Rinv, int r) {
    const int lane = threadIdx.x & 31;
    double g[RMAX], x[RMAX], invd[RMAX];
#pragma unroll
    for (int i = 0; i < RMAX; i++) g[i] = (i < r && lane < r) ? G[i * r + lane] : 0.0;
    const double g00 = __shfl_sync(0xffffffffu, g[0], 0);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < RMAX; k++) {
        if (k >= r) break;
        const double d = __shfl_sync(0xffffffffu, g[k], k);
        if (!(d > 1e-28 * g00)) ok = false;
        const double rkk = sqrt(fmax(d, 1e-300));
        const double inv = 1.0 / rkk;
        invd[k] = inv;
        if (lane > k) g[k] *= inv;
        if (lane == k) g[k] = rkk;
#pragma unroll
        for (int i = k + 1; i < RMAX; i++) {
            if (i >= r) break;
            const double rki = __shfl_sync(0xffffffffu, g[k], i);
            if (lane >= i) g[i] = fma(-rki, g[k], g[i]);
        }
    }
    if constexpr (!INV) {
        if (lane < r) {
#pragma unroll
            for (int i = 0; i < RMAX; i++)
                if (i < r) G[i * r + lane] = i <= lane ? g[i] : 0.0;
        }
        __syncwarp();
        return ok;
    } else {
        // Column `lane` of R^{-1} by back substitution; x[j] = 0 for j > lane.
#pragma unroll
        for (int i = 0; i < RMAX; i++) x[i] = (i == lane) ? invd[i] : 0.0;
#pragma unroll
        for (int i = RMAX - 2; i >= 0; i--) {
            if (i >= r - 1) continue;
            double sacc = 0.0;
#pragma unroll
            for (int j = i + 1; j < RMAX; j++) {
                if (j >= r) break;
                const double rij = __shfl_sync(0xffffffffu, g[i], j);
                sacc = fma(rij, x[j], sacc);
            }
            if (i < lane) x[i] = -sacc * invd[i];
        }
        if (lane < r) {
#pragma unroll
            for (int i = 0; i < RMAX; i++)
                if (i < r) {
                    Rinv[i * r + lane] = x[i];
                    G[i * r + lane] = i <= lane ? g[i] : 0.0;
                }
        }
        __syncwarp();
        return ok;
    }
}

// Subspace iteration L <- orth(S L), `iters` times, one CTA.  S (n x n,
// symmetric) is staged in shared memory -- whole when it fits, as its packed
// upper triangle for n up to ~220, else read from L2.  L and Z (n x r) live in
// shared memory when they fit.  Intermediate steps orthonormalise with one
// CholeskyQR pass (only conditioning matters there), the last step with two
// (CholeskyQR2, orthonormal to FP64 rounding); a Cholesky breakdown
// (rank-deficient S L) switches that step to Householder.
enum { S_GLOBAL = 0, S_FULL = 1, S_PACKED = 2 };

__device__ __forceinline__ double s_at(const double *S, int64_t n, int mode, int64_t i,
                                       int64_t k) {
    if (mode == S_PACKED) {
        const int64_t a = i < k ? i : k, b = i < k ? k : i;
        return S[a + b * (b + 1) / 2];
    }
    return S[i + n * k];
}

// Forward substitution Q[i, :] = Z[i, :] R^{-1} for every row i (R upper,
// row-major r x r in smem, Rinv_diag its reciprocal diagonal), one thread per
// row: the r-step chain runs on 96+ rows at once instead of one warp.
__device__ __forceinline__ void rows_trsm(const double *Z, double *Q, int64_t n, int64_t r,
                                          const double *R) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        double q[32];
#pragma unroll
        for (int c = 0; c < 32; c++) {
            if (c >= r) break;
            double acc = Z[i + c * n];
#pragma unroll
            for (int k = 0; k < 32; k++) {
                if (k >= c) break;
                acc = fma(-q[k], R[k * r + c], acc);
            }
            q[c] = acc / R[c * r + c];
            Q[i + c * n] = q[c];
        }
    }
}

template <int RMAX>
__global__ void __launch_bounds__(LA_NT) subspace_kernel(const double *Sg, int64_t n,
                                                         double *Lg, int64_t r, int iters,
                                                         double *work, int s_mode,
                                                         int zl_in_smem, int *flag) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[33];
    __shared__ int bad;
    const int t = threadIdx.x;
    double *G = sm;                // r*r
    double *Ri = sm + r * r;       // r*r (unused scratch for the Cholesky helper)
    double *cur = sm + 2 * r * r;  // after the two r x r blocks
    const double *S = Sg;
    if (s_mode == S_FULL) {
        double *Ss = cur;
        for (int64_t e = t; e < n * n; e += blockDim.x) Ss[e] = Sg[e];
        S = Ss;
        cur += n * n;
    } else if (s_mode == S_PACKED) {
        double *Ss = cur;
        const int64_t np = n * (n + 1) / 2;
        for (int64_t e = t; e < n * n; e += blockDim.x) {
            const int64_t i = e % n, k = e / n;
            if (i <= k) Ss[i + k * (k + 1) / 2] = Sg[e];
        }
        S = Ss;
        cur += (np + 1) & ~int64_t(1);
    }
    double *L, *Z;
    if (zl_in_smem) {
        L = cur;
        Z = cur + n * r;
    } else {
        L = work;
        Z = work + n * r;
    }
    double *hwork = work + 2 * n * r;  // n*r + r for the Householder fallback
    for (int64_t e = t; e < n * r; e += blockDim.x) L[e] = Lg[e];
    __syncthreads();
    const int64_t cgroups = (r + 3) / 4;
    const int npairs = (int)(r * (r + 1) / 2);

    // One CholeskyQR pass: dst = orth(src) through G = src^T src = R^T R.
    auto cholqr = [&](const double *src, double *dst) -> bool {
        for (int task = t; task < 4 * ((npairs + 7) / 8) * 8; task += blockDim.x) {
            const int pr = task >> 2, part = task & 3;
            double sacc = 0.0;
            int a = 0, b = 0;
            if (pr < npairs) {
                int rem = pr;
                while (rem >= (int)r - a) {
                    rem -= (int)r - a;
                    a++;
                }
                b = a + rem;
                const double *ca = src + (int64_t)a * n, *cb = src + (int64_t)b * n;
                for (int64_t k = part; k < n; k += 4) sacc = fma(ca[k], cb[k], sacc);
            }
            sacc += __shfl_xor_sync(0xffffffffu, sacc, 1);
            sacc += __shfl_xor_sync(0xffffffffu, sacc, 2);
            if (pr < npairs && part == 0) {
                G[a * r + b] = sacc;
                G[b * r + a] = sacc;
            }
        }
        __syncthreads();
        if (t < 32) {
            const bool ok = warp_chol_inv<RMAX, false>(G, Ri, (int)r);
            if (t == 0) bad = ok ? 0 : 1;
        }
        __syncthreads();
        if (bad) return false;
        rows_trsm(src, dst, n, r, G);
        __syncthreads();
        return true;
    };

    // span(S^iters L): products Z <- S Z, orthonormalised after the second
    // product (conditioning stays within (l1/lr)^2) and at the end (two passes).
    bool broke = false;
    double *cur_in = L, *cur_out = Z;
    for (int it = 0; it < iters && !broke; it++) {
        for (int64_t task = t; task < n * cgroups; task += blockDim.x) {
            const int64_t i = task % n, c0 = 4 * (task / n);
            double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
            const double *l0 = cur_in + c0 * n;
            const bool h1 = c0 + 1 < r, h2 = c0 + 2 < r, h3 = c0 + 3 < r;
#pragma unroll 4
            for (int64_t k = 0; k < n; k++) {
                const double sv = s_at(S, n, s_mode, i, k);
                a0 = fma(sv, l0[k], a0);
                if (h1) a1 = fma(sv, l0[k + n], a1);
                if (h2) a2 = fma(sv, l0[k + 2 * n], a2);
                if (h3) a3 = fma(sv, l0[k + 3 * n], a3);
            }
            cur_out[i + c0 * n] = a0;
            if (h1) cur_out[i + (c0 + 1) * n] = a1;
            if (h2) cur_out[i + (c0 + 2) * n] = a2;
            if (h3) cur_out[i + (c0 + 3) * n] = a3;
        }
        __syncthreads();
        double *tmp = cur_in;
        cur_in = cur_out;
        cur_out = tmp;
        const bool last = it == iters - 1;
        if (last || (it % 2) == 1) {
            // cur_in holds the product; orthonormalise into cur_out, then back.
            if (!cholqr(cur_in, cur_out)) {
                broke = true;
                break;
            }
            if (last) {
                if (!cholqr(cur_out, cur_in)) {
                    broke = true;
                    break;
                }
            } else {
                tmp = cur_in;
                cur_in = cur_out;
                cur_out = tmp;
            }
        }
    }
    if (broke) {
        // Rank-deficient or badly conditioned: restart from the caller's L and
        // run every step with Householder orthonormalisation.
        for (int64_t e = t; e < n * r; e += blockDim.x) L[e] = Lg[e];
        __syncthreads();
        for (int it = 0; it < iters; it++) {
            for (int64_t e = t; e < n * r; e += blockDim.x) {
                const int64_t i = e % n, c = e / n;
                double acc = 0.0;
                for (int64_t k = 0; k < n; k++) acc = fma(s_at(S, n, s_mode, i, k), L[k + c * n], acc);
                hwork[e] = acc;
            }
            __syncthreads();
            hqr_device(hwork, n, r, hwork + n * r, L, red);
            __syncthreads();
        }
        if (t == 0 && flag) atomicOr(flag, 2);
        for (int64_t e = t; e < n * r; e += blockDim.x) Lg[e] = L[e];
        return;
    }
    for (int64_t e = t; e < n * r; e += blockDim.x) Lg[e] = cur_in[e];
}

// ---------------------------------------------------------------------------
// Subspace iteration on the FP64 tensor-core path (mma.sync m8n8k4 .f64) for
// n <= 256 and r <= RT (8, 16 or 32), one CTA of 8 warps.  Same schedule as
// subspace_kernel (five products S Z, CholeskyQR after the 2nd and 4th,
// CholeskyQR2 after the 5th).  Shared-memory layout:
//  * S col-major with a leading dimension LDS = 4 (mod 16) and Z, Q row-major
//    n8 x RT with pitch RT + 4: the 8 x 4 and 4 x 8 operand fragments then hit
//    16 distinct 8-byte bank pairs per half-warp;
//  * rows n..n8-1 and columns r..RT-1 are zero padding, so every product,
//    Gram and solve runs on whole 8 x 8 tiles.
// S Z and Z R^{-1}: each warp owns whole m-tile rows (all RT/8 n-tiles, two
// m-tiles interleaved).  Z^T Z: whole K split over warps when it has fewer
// than 8 tiles, partials summed in a fixed order.  Cholesky and R^{-1} in
// warp 0 (rsqrt per pivot, multiplications by the reciprocal diagonal).  A
// Cholesky breakdown restarts from the caller's L with Householder steps.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void la_cp_async16(void *smem, const void *gmem) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void la_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void la_cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

constexpr int SM_WARPS = 8;
constexpr int SM_NT = SM_WARPS * 32;
constexpr int SM_GP = 512;  // doubles of Gram partials (K split only below 8 tiles)

__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int RT>
struct SmTile {
    static constexpr int LDQ = RT + 4;  // Z / Q pitch (= 4 mod 16 for RT in {16, 32}; 12 for 8)
    static constexpr int LDR = RT + 4;  // R^{-1} pitch
    static constexpr int NT = RT / 8;   // n-tiles
};

__host__ __device__ inline int sm_lds(int n8) { return ((n8 + 11) / 16) * 16 + 4; }

// dst = S src   (n8 x RT), S from shared (ld lds) or from global (ld n).
template <int RT, int SMODE>
__device__ __forceinline__ void sm_product(const double *Ss, int lds, const double *__restrict__ Sg,
                                           int n, int n8, const double *src, double *dst) {
    using T = SmTile<RT>;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int mtiles = n8 / 8, ksteps = (n + 3) / 4;
    for (int mt0 = w; mt0 < mtiles; mt0 += 2 * SM_WARPS) {
        const int mt1 = mt0 + SM_WARPS;
        const bool two = mt1 < mtiles;
        double acc[2][T::NT][2];
#pragma unroll
        for (int m = 0; m < 2; m++)
#pragma unroll
            for (int j = 0; j < T::NT; j++) acc[m][j][0] = acc[m][j][1] = 0.0;
        const int i0 = 8 * mt0 + g, i1 = 8 * mt1 + g;
#pragma unroll 4
        for (int kk = 0; kk < ksteps; kk++) {
            const int k = 4 * kk + t;
            double a0, a1 = 0.0;
            if (SMODE == S_FULL) {
                a0 = Ss[i0 + lds * k];
                if (two) a1 = Ss[i1 + lds * k];
            } else {
                a0 = (i0 < n && k < n) ? __ldg(Sg + i0 + (int64_t)n * k) : 0.0;
                if (two) a1 = (i1 < n && k < n) ? __ldg(Sg + i1 + (int64_t)n * k) : 0.0;
            }
#pragma unroll
            for (int j = 0; j < T::NT; j++) {
                const double b = src[k * T::LDQ + 8 * j + g];
                dmma884(acc[0][j][0], acc[0][j][1], a0, b);
                if (two) dmma884(acc[1][j][0], acc[1][j][1], a1, b);
            }
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
            if (m == 1 && !two) break;
            const int row = 8 * (m ? mt1 : mt0) + g;
#pragma unroll
            for (int j = 0; j < T::NT; j++)
                *reinterpret_cast<double2 *>(dst + row * T::LDQ + 8 * j + 2 * t) =
                    make_double2(acc[m][j][0], acc[m][j][1]);
        }
    }
}

// dst = src Ri   (n8 x RT times RT x RT upper).
template <int RT>
__device__ __forceinline__ void sm_apply(const double *src, const double *Ri, int n8,
                                         double *dst) {
    using T = SmTile<RT>;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int mtiles = n8 / 8;
    for (int mt = w; mt < mtiles; mt += SM_WARPS) {
        double acc[T::NT][2];
#pragma unroll
        for (int j = 0; j < T::NT; j++) acc[j][0] = acc[j][1] = 0.0;
        const int row = 8 * mt + g;
#pragma unroll
        for (int kk = 0; kk < RT / 4; kk++) {
            const double a = src[row * T::LDQ + 4 * kk + t];
#pragma unroll
            for (int j = 0; j < T::NT; j++)
                dmma884(acc[j][0], acc[j][1], a, Ri[(4 * kk + t) * T::LDR + 8 * j + g]);
        }
#pragma unroll
        for (int j = 0; j < T::NT; j++)
            *reinterpret_cast<double2 *>(dst + row * T::LDQ + 8 * j + 2 * t) =
                make_double2(acc[j][0], acc[j][1]);
    }
}

// G = src^T src (RT x RT row-major); rows/columns >= r replaced by the identity.
template <int RT>
__device__ __forceinline__ void sm_gram(const double *src, int n, int r, double *Gp, double *G) {
    using T = SmTile<RT>;
    constexpr int TILES = T::NT * T::NT;
    constexpr int KSP = TILES >= SM_WARPS ? 1 : SM_WARPS / TILES;
    static_assert(KSP == 1 || KSP * RT * RT <= SM_GP, "Gram partials");
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int ksteps = (n + 3) / 4;
    if (KSP == 1) {
        for (int tt = w; tt < TILES; tt += SM_WARPS) {
            const int ta = tt % T::NT, tb = tt / T::NT;
            double d0 = 0.0, d1 = 0.0;
            for (int kk = 0; kk < ksteps; kk++) {
                const int k = 4 * kk + t;
                dmma884(d0, d1, src[k * T::LDQ + 8 * ta + g], src[k * T::LDQ + 8 * tb + g]);
            }
            const int a = 8 * ta + g, b = 8 * tb + 2 * t;
            G[a * RT + b] = d0;
            G[a * RT + b + 1] = d1;
        }
        __syncthreads();
    } else {
        const int tt = w % TILES, part = w / TILES;
        const int ta = tt % T::NT, tb = tt / T::NT;
        double d0 = 0.0, d1 = 0.0;
        for (int kk = part; kk < ksteps; kk += KSP) {
            const int k = 4 * kk + t;
            dmma884(d0, d1, src[k * T::LDQ + 8 * ta + g], src[k * T::LDQ + 8 * tb + g]);
        }
        const int a = 8 * ta + g, b = 8 * tb + 2 * t;
        Gp[part * RT * RT + a * RT + b] = d0;
        Gp[part * RT * RT + a * RT + b + 1] = d1;
        __syncthreads();
        for (int e = threadIdx.x; e < RT * RT; e += SM_NT) {
            double s = 0.0;
#pragma unroll
            for (int p = 0; p < KSP; p++) s += Gp[p * RT * RT + e];
            G[e] = s;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < RT * RT; e += SM_NT) {
        const int a = e / RT, b = e % RT;
        if (a >= r || b >= r) G[e] = (a == b) ? 1.0 : 0.0;
    }
    __syncthreads();
}

// G = R^T R (R upper, overwriting the upper triangle of G; the strict lower
// triangle is zeroed), with the whole CTA: per pivot k every thread reads the
// pivot and row k, then the threads owning entries (i, j), k < i <= j, update
// them while the owners of row k scale it.  Two barriers per pivot, no
// divides.  dinv[k] = 1 / R(k, k) (1 for the padding).  Returns false on a
// non-positive pivot (the same value in every thread).
template <int RT>
__device__ __forceinline__ bool sm_chol(double *G, double *dinv, int r) {
    constexpr int EPT = (RT * RT + SM_NT - 1) / SM_NT;
    const int t = threadIdx.x;
    const double g00 = G[0];
    bool ok = g00 > 0.0;
    for (int k = 0; k < r; k++) {
        const double d = G[k * RT + k];
        ok = ok && (d > 1e-28 * g00);
        const double ri = rsqrt(fmax(d, 1e-300));
        double upd[EPT];
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            const int e = t + q * SM_NT, i = e / RT, j = e % RT;
            upd[q] = (e < RT * RT && i > k && i <= j && j < r)
                         ? (G[k * RT + i] * ri) * (G[k * RT + j] * ri)
                         : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            const int e = t + q * SM_NT, i = e / RT, j = e % RT;
            if (e < RT * RT && j < r) {
                if (i > k && i <= j) G[e] -= upd[q];
                else if (i == k && j >= k) G[e] *= ri;
            }
        }
        if (t == k) dinv[k] = ri;
        __syncthreads();
    }
    for (int e = t; e < RT * RT; e += SM_NT) {
        const int i = e / RT, j = e % RT;
        if (i > j) G[e] = 0.0;
    }
    if (t >= r && t < RT) dinv[t] = 1.0;
    __syncthreads();
    return ok;
}

// Warp 0: Ri = R^{-1} (row-major, pitch LDR) from R in the upper triangle of G
// and dinv.  Lane c solves column c: x_i = (delta_{i,c} - sum_{j>i} R(i,j) x_j) dinv_i.
template <int RT>
__device__ __forceinline__ void sm_rinv(const double *G, double *Ri, const double *dinv) {
    constexpr int LDR = SmTile<RT>::LDR;
    const int lane = threadIdx.x & 31;
    double x[RT];
#pragma unroll
    for (int i = RT - 1; i >= 0; i--) {
        double s0 = (i == lane) ? 1.0 : 0.0, s1 = 0.0;
#pragma unroll
        for (int j = i + 1; j < RT; j++) {
            const double rij = G[i * RT + j];
            if (j & 1)
                s1 = fma(-rij, x[j], s1);
            else
                s0 = fma(-rij, x[j], s0);
        }
        x[i] = (s0 + s1) * dinv[i];
    }
    if (lane < RT) {
#pragma unroll
        for (int i = 0; i < RT; i++) Ri[i * LDR + lane] = i <= lane ? x[i] : 0.0;
    }
}

// Cholesky + R^{-1} (all threads call it; ends with a barrier).
template <int RT>
__device__ __forceinline__ bool sm_chol_inv(double *G, double *Ri, double *dinv, int r) {
    const bool ok = sm_chol<RT>(G, dinv, r);
    if (threadIdx.x < 32) sm_rinv<RT>(G, Ri, dinv);
    __syncthreads();
    return ok;
}

// After one CholeskyQR pass, Q^T Q = I + E with E tiny.  When max |E| <= 1e-8,
// C = I - E/2 + 3E^2/8 (the series of (I + E)^{-1/2}) makes Q C orthonormal to
// rounding; C goes to Ri (pitch LDR) for sm_apply.  Returns false when E is too
// large, and the caller runs a second CholeskyQR pass instead.  All threads.
template <int RT>
__device__ __forceinline__ bool sm_polar_fix(const double *G, double *Ri, double *red) {
    constexpr int LDR = SmTile<RT>::LDR;
    const int t = threadIdx.x;
    double emax = 0.0;
    for (int e = t; e < RT * RT; e += SM_NT) {
        const int a = e / RT, b = e % RT;
        emax = fmax(emax, fabs(G[e] - (a == b ? 1.0 : 0.0)));
    }
    for (int o = 16; o > 0; o >>= 1) emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    if ((t & 31) == 0) red[t >> 5] = emax;
    __syncthreads();
    double m = 0.0;
#pragma unroll
    for (int w = 0; w < SM_WARPS; w++) m = fmax(m, red[w]);
    if (!(m <= 1e-8)) {
        __syncthreads();
        return false;
    }
    for (int e = t; e < RT * RT; e += SM_NT) {
        const int a = e / RT, b = e % RT;
        double e2 = 0.0;
#pragma unroll
        for (int k = 0; k < RT; k++)
            e2 = fma(G[a * RT + k] - (a == k ? 1.0 : 0.0), G[k * RT + b] - (k == b ? 1.0 : 0.0), e2);
        const double eab = G[e] - (a == b ? 1.0 : 0.0);
        Ri[a * LDR + b] = (a == b ? 1.0 : 0.0) - 0.5 * eab + 0.375 * e2;
    }
    __syncthreads();
    return true;
}

template <int RT>
__host__ __device__ inline size_t sm_smem_doubles(int n, bool s_in_smem) {
    const int n8 = (n + 7) / 8 * 8;
    size_t d = 2 * (size_t)n8 * SmTile<RT>::LDQ   // Z, Q
               + (size_t)SM_GP                    // Gram partials
               + (size_t)RT * RT                  // G / R
               + (size_t)RT * SmTile<RT>::LDR     // R^{-1}
               + 32;                              // dinv
    if (s_in_smem) d += (size_t)sm_lds(n8) * n8;
    return d;
}

template <int RT, int SMODE>
__global__ void __launch_bounds__(SM_NT, 1) subspace_mma_kernel(const double *Sg, int n,
                                                             double *Lg, int r, int iters,
                                                             double *work, int *flag) {
    using T = SmTile<RT>;
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[33];
    __shared__ int bad;
    const int t = threadIdx.x;
    pdl_wait();
    const int n8 = (n + 7) / 8 * 8;
    const int lds = sm_lds(n8);
    double *A = sm;
    double *B = A + n8 * T::LDQ;
    double *Gp = B + n8 * T::LDQ;
    double *G = Gp + SM_GP;
    double *Ri = G + RT * RT;
    double *dinv = Ri + RT * T::LDR;
    double *Ss = dinv + 32;
    if (SMODE == S_FULL) {
        // S goes global -> shared with asynchronous 16-byte copies (one
        // latency for the whole matrix); the padding is zeroed meanwhile.
        if ((n & 1) == 0) {
            const int hc = n / 2;
            for (int e = t; e < hc * n; e += SM_NT) {
                const int k = e / hc, q = e - k * hc;
                la_cp_async16(Ss + lds * k + 2 * q, Sg + (int64_t)n * k + 2 * q);
            }
            la_cp_commit();
        } else {
            for (int e = t; e < n * n; e += SM_NT) {
                const int k = e / n, i = e - k * n;
                Ss[i + lds * k] = Sg[e];
            }
        }
        const int pr = lds - n;
        for (int e = t; e < pr * n8; e += SM_NT) {
            const int k = e / pr, i = n + (e - k * pr);
            Ss[i + lds * k] = 0.0;
        }
        for (int e = t; e < (n8 - n) * n; e += SM_NT) {
            const int k = n + e / n, i = e % n;
            Ss[i + lds * k] = 0.0;
        }
    }
    // L (n x r col-major) -> A (row-major, pitch LDQ, zero padded): all loads
    // of a thread are issued before its stores.
    for (int e = t; e < n8 * T::LDQ; e += SM_NT) {
        A[e] = 0.0;
        B[e] = 0.0;
    }
    __syncthreads();
    {
        constexpr int MAXQ = 32;  // n * r <= 256 * 32 = SM_NT * MAXQ
        double v[MAXQ];
#pragma unroll
        for (int q = 0; q < MAXQ; q++) {
            const int e = t + SM_NT * q;
            v[q] = e < n * r ? Lg[e] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < MAXQ; q++) {
            const int e = t + SM_NT * q;
            if (e < n * r) {
                const int c = e / n, i = e - c * n;
                A[i * T::LDQ + c] = v[q];
            }
        }
    }
    if (SMODE == S_FULL && (n & 1) == 0) la_cp_wait_all();
    if (t == 0) bad = 0;
    __syncthreads();

    double *cur = A, *oth = B;
    for (int it = 0; it < iters; it++) {
        sm_product<RT, SMODE>(Ss, lds, Sg, n, n8, cur, oth);
        __syncthreads();
        double *tmp = cur;
        cur = oth;
        oth = tmp;
        const bool last = it == iters - 1;
        if (last || (it & 1)) {
            const int passes = last ? 2 : 1;
            for (int p = 0; p < passes; p++) {
                sm_gram<RT>(cur, n, r, Gp, G);
                // The second pass is usually a tiny correction (polar fix).
                if (!(p == 1 && sm_polar_fix<RT>(G, Ri, red))) {
                    if (!sm_chol_inv<RT>(G, Ri, dinv, r)) {
                        bad = 1;
                        break;
                    }
                }
                sm_apply<RT>(cur, Ri, n8, oth);
                __syncthreads();
                tmp = cur;
                cur = oth;
                oth = tmp;
            }
            if (bad) break;
        }
    }
    // Dependents launch once the iteration is done (launched at the start,
    // they took SM slots for the whole kernel; about 1 % of a decomposition).
    pdl_trigger();
    if (!bad) {
        for (int e = t; e < n * r; e += SM_NT) {
            const int i = e % n, c = e / n;
            Lg[e] = cur[i * T::LDQ + c];
        }
        return;
    }
    // Rank-deficient or badly conditioned: restart from the caller's L and run
    // every step with Householder orthonormalisation (col-major, in `work`).
    double *Lw = work, *hw = work + 2 * (int64_t)n * r;
    for (int e = t; e < n * r; e += SM_NT) Lw[e] = Lg[e];
    __syncthreads();
    for (int it = 0; it < iters; it++) {
        for (int e = t; e < n * r; e += SM_NT) {
            const int i = e % n, c = e / n;
            double acc = 0.0;
            for (int k = 0; k < n; k++) {
                const double sv = SMODE == S_FULL ? Ss[i + lds * k] : __ldg(Sg + i + (int64_t)n * k);
                acc = fma(sv, Lw[k + n * c], acc);
            }
            hw[e] = acc;
        }
        __syncthreads();
        hqr_device(hw, n, r, hw + (int64_t)n * r, Lw, red);
        __syncthreads();
    }
    if (t == 0 && flag) atomicOr(flag, 2);
    for (int e = t; e < n * r; e += SM_NT) Lg[e] = Lw[e];
}

// Q[b] = orth(A[b]) for a batch of m x n (n <= RT) col-major matrices, one CTA
// each: CholeskyQR2 with the mma.sync Gram / apply above; a Cholesky
// breakdown falls back to Householder on work[b] (m n + n doubles).  The span
// is that of A, as with Householder QR; the basis may differ by a rotation.
template <int RT>
__global__ void __launch_bounds__(SM_NT, 1) cholqr2_batch_kernel(const double *const *A,
                                                                double *const *Q,
                                                                const int64_t *m,
                                                                const int64_t *n,
                                                                double *const *work) {
    using T = SmTile<RT>;
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[33];
    __shared__ int bad;
    const int b = blockIdx.x, t = threadIdx.x;
    const int M = (int)m[b], r = (int)n[b];
    const int M8 = (M + 7) / 8 * 8;
    double *Z0 = sm;
    double *Z1 = Z0 + M8 * T::LDQ;
    double *Gp = Z1 + M8 * T::LDQ;
    double *G = Gp + SM_GP;
    double *Ri = G + RT * RT;
    double *dinv = Ri + RT * T::LDR;
    for (int e = t; e < M8 * T::LDQ; e += SM_NT) {
        const int i = e / T::LDQ, c = e % T::LDQ;
        Z0[e] = (i < M && c < r) ? A[b][i + (int64_t)M * c] : 0.0;
    }
    if (t == 0) bad = 0;
    __syncthreads();
    double *cur = Z0, *oth = Z1;
    for (int p = 0; p < 2; p++) {
        sm_gram<RT>(cur, M, r, Gp, G);
        if (!sm_chol_inv<RT>(G, Ri, dinv, r)) {
            bad = 1;
            break;
        }
        sm_apply<RT>(cur, Ri, M8, oth);
        __syncthreads();
        double *tmp = cur;
        cur = oth;
        oth = tmp;
    }
    if (!bad) {
        for (int e = t; e < M * r; e += SM_NT) {
            const int i = e % M, c = e / M;
            Q[b][e] = cur[i * T::LDQ + c];
        }
        return;
    }
    double *W = work[b];
    for (int e = t; e < M * r; e += SM_NT) W[e] = A[b][e];
    __syncthreads();
    hqr_device(W, M, r, W + (int64_t)M * r, Q[b], red);
}

template <int RT, int SMODE>
void launch_subspace_mma(dt_ctx *ctx, const double *S, int n, double *L, int r, int iters,
                         double *work, int *flag) {
    const size_t smem = sm_smem_doubles<RT>(n, SMODE == S_FULL) * sizeof(double);
    auto kern = subspace_mma_kernel<RT, SMODE>;
    smem_limit(ctx, kern, smem);
    DT_LAUNCH_PDL(ctx, kern, 1, SM_NT, smem, S, n, L, r, iters, work, flag);
}

template <int RT>
void subspace_mma(dt_ctx *ctx, const double *S, int n, double *L, int r, int iters,
                  double *work, int *flag) {
    if (sm_smem_doubles<RT>(n, true) * sizeof(double) <= 220 * 1024)
        launch_subspace_mma<RT, S_FULL>(ctx, S, n, L, r, iters, work, flag);
    else
        launch_subspace_mma<RT, S_GLOBAL>(ctx, S, n, L, r, iters, work, flag);
}

// Subspace iteration for ranks above 32: Householder QR every step, S, L and Z
// in global memory (L2-resident).  work >= 3*n*r + r.
__global__ void __launch_bounds__(LA_NT) subspace_wide_kernel(const double *S, int64_t n,
                                                              double *L, int64_t r, int iters,
                                                              double *work) {
    __shared__ double red[33];
    double *Z = work, *W = work + n * r, *tau = work + 2 * n * r;
    for (int it = 0; it < iters; it++) {
        for (int64_t e = threadIdx.x; e < n * r; e += blockDim.x) {
            const int64_t i = e % n, c = e / n;
            double acc = 0.0;
            for (int64_t k = 0; k < n; k++) acc = fma(S[i + n * k], L[k + n * c], acc);
            Z[e] = acc;
        }
        __syncthreads();
        for (int64_t e = threadIdx.x; e < n * r; e += blockDim.x) W[e] = Z[e];
        __syncthreads();
        hqr_device(W, n, r, tau, L, red);
        __syncthreads();
    }
}

// LU with partial pivoting on W (n x n col-major copy of A), then Ainv by
// solving for the identity columns.
__global__ void __launch_bounds__(LA_NT) lu_inverse_kernel(const double *A, int64_t n,
                                                           double *Ainv, double *W,
                                                           int *flag) {
    __shared__ double red_v[32];
    __shared__ int red_i[32];
    __shared__ int piv_row;
    extern __shared__ int perm[];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int64_t e = t; e < n * n; e += blockDim.x) W[e] = A[e];
    for (int64_t i = t; i < n; i += blockDim.x) perm[i] = (int)i;
    __syncthreads();
    for (int64_t k = 0; k < n; k++) {
        double best = -1.0;
        int bi = (int)k;
        for (int64_t i = k + t; i < n; i += blockDim.x) {
            const double v = fabs(W[i + k * n]);
            if (v > best) {
                best = v;
                bi = (int)i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            red_v[warp] = best;
            red_i[warp] = bi;
        }
        __syncthreads();
        if (t == 0) {
            double bv = -1.0;
            int bb = (int)k;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++)
                if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bb)) {
                    bv = red_v[w];
                    bb = red_i[w];
                }
            piv_row = bb;
            if (!(bv > 0.0)) atomicOr(flag, 1);
        }
        __syncthreads();
        const int p = piv_row;
        if (p != k) {
            for (int64_t c = t; c < n; c += blockDim.x) {
                const double tmp = W[k + c * n];
                W[k + c * n] = W[p + c * n];
                W[p + c * n] = tmp;
            }
            if (t == 0) {
                const int tp = perm[k];
                perm[k] = perm[p];
                perm[p] = tp;
            }
        }
        __syncthreads();
        const double d = W[k + k * n];
        for (int64_t i = k + 1 + t; i < n; i += blockDim.x) W[i + k * n] /= d;
        __syncthreads();
        for (int64_t e = t; e < (n - k - 1) * (n - k - 1); e += blockDim.x) {
            const int64_t i = k + 1 + e % (n - k - 1), c = k + 1 + e / (n - k - 1);
            W[i + c * n] = fma(-W[i + k * n], W[k + c * n], W[i + c * n]);
        }
        __syncthreads();
    }
    // Solve L U x = P e_c for every column c (one thread per column).
    for (int64_t c = t; c < n; c += blockDim.x) {
        double *x = Ainv + c * n;
        for (int64_t i = 0; i < n; i++) {
            double s = (perm[i] == c) ? 1.0 : 0.0;
            for (int64_t j = 0; j < i; j++) s = fma(-W[i + j * n], x[j], s);
            x[i] = s;
        }
        for (int64_t i = n - 1; i >= 0; i--) {
            double s = x[i];
            for (int64_t j = i + 1; j < n; j++) s = fma(-W[i + j * n], x[j], s);
            x[i] = s / W[i + i * n];
        }
    }
}

// Householder QR of several small matrices at once (one CTA each, 128
// threads so the per-column barriers stay cheap): Q[b] = Q of A[b].
__global__ void __launch_bounds__(128) hqr_batch_kernel(const double *const *A,
                                                         double *const *Q, const int64_t *m,
                                                         const int64_t *n, double *const *work) {
    __shared__ double red[33];
    const int b = blockIdx.x;
    const int64_t mb = m[b], nb = n[b];
    double *W = work[b];
    for (int64_t e = threadIdx.x; e < mb * nb; e += blockDim.x) W[e] = A[b][e];
    __syncthreads();
    hqr_device(W, mb, nb, W + mb * nb, Q[b], red);
}

// Cholesky of the r x r SPD G (col-major) and L^{-1} (lower) for the row
// orthonormalisation; one CTA, r small.  Output Linv col-major.
__global__ void chol_lower_inv_kernel(const double *Gg, int r, double *Linv, int *flag) {
    extern __shared__ double sm[];
    double *G = sm, *Ri = sm + r * r;
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) G[e] = Gg[e];  // symmetric
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool ok = warp_chol_inv<32>(G, Ri, r);
        if (!ok && threadIdx.x == 0) atomicOr(flag, 1);
    }
    __syncthreads();
    // G = R^T R with R upper; L = R^T, so L^{-1} = (R^{-1})^T.
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int i = e % r, c = e / r;  // Linv(i, c) = Rinv(c, i)
        Linv[e] = Ri[c * r + i];
    }
}

// Row Gram on the FP64 tensor cores (mma.sync m8n8k4): A is r x m col-major
// (factor row k = column k), G = sum_k a_k a_k^T.  With 4 columns per k-step,
// the fragment A[g][t] = a_{4kk+t}(8h + g) is also the B fragment B[t][g] of
// tile h, so each lane loads TT values per k-step for TT x TT MMAs.  Warps of
// a block take interleaved k-steps of the block's column range; tiles are
// summed over the warps in a fixed order into part[block][r*r].
template <int RT>
__global__ void __launch_bounds__(256) rows_gram_mma_kernel(const double *__restrict__ A, int r,
                                                            int64_t m, int64_t cols_per_block,
                                                            double *__restrict__ part) {
    constexpr int TT = RT / 8;
    __shared__ double red[4][RT * RT];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int64_t k0 = blockIdx.x * cols_per_block;
    const int64_t k1 = min(m, k0 + cols_per_block);
    double acc[TT][TT][2];
#pragma unroll
    for (int a = 0; a < TT; a++)
#pragma unroll
        for (int b = 0; b < TT; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll 4
    for (int64_t c0 = k0 + 4 * w; c0 < k1; c0 += 32) {
        const int64_t col = c0 + t;
        double f[TT];
#pragma unroll
        for (int h = 0; h < TT; h++)
            f[h] = (col < k1 && 8 * h + g < r) ? A[col * r + 8 * h + g] : 0.0;
#pragma unroll
        for (int a = 0; a < TT; a++)
#pragma unroll
            for (int b = 0; b < TT; b++) {
                asm volatile(
                    "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                    : "+d"(acc[a][b][0]), "+d"(acc[a][b][1])
                    : "d"(f[a]), "d"(f[b]));
            }
    }
    // Warps 0-3 store, warps 4-7 add theirs (fixed order), then 4 slots sum.
    if (w < 4) {
#pragma unroll
        for (int a = 0; a < TT; a++)
#pragma unroll
            for (int b = 0; b < TT; b++)
#pragma unroll
                for (int q = 0; q < 2; q++)
                    red[w][(8 * a + g) * RT + 8 * b + 2 * t + q] = acc[a][b][q];
    }
    __syncthreads();
    if (w >= 4) {
#pragma unroll
        for (int a = 0; a < TT; a++)
#pragma unroll
            for (int b = 0; b < TT; b++)
#pragma unroll
                for (int q = 0; q < 2; q++)
                    red[w - 4][(8 * a + g) * RT + 8 * b + 2 * t + q] += acc[a][b][q];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int i = e / r, j = e - i * r;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 4; q++) s += red[q][i * RT + j];
        part[(int64_t)blockIdx.x * r * r + i * r + j] = s;
    }
}

// T = Linv A on the FP64 tensor cores: Linv (r x r lower, col-major) is the A
// operand (held in registers), 8-column blocks of A (r x m col-major) the B
// operand; one warp per 8-column block.
template <int RT>
__global__ void __launch_bounds__(256) rows_apply_mma_kernel(const double *__restrict__ A, int r,
                                                             int64_t m,
                                                             const double *__restrict__ Linv,
                                                             double *__restrict__ T) {
    constexpr int TT = RT / 8, KS = RT / 4;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    double la[TT][KS];
#pragma unroll
    for (int h = 0; h < TT; h++)
#pragma unroll
        for (int kk = 0; kk < KS; kk++) {
            const int i = 8 * h + g, c = 4 * kk + t;
            la[h][kk] = (i < r && c < r) ? Linv[i + (int64_t)r * c] : 0.0;
        }
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nblk = (m + 7) / 8;
    for (int64_t cb = warp0; cb < nblk; cb += nwarps) {
        double acc[TT][2];
#pragma unroll
        for (int h = 0; h < TT; h++) acc[h][0] = acc[h][1] = 0.0;
        const int64_t colb = 8 * cb + g;
#pragma unroll
        for (int kk = 0; kk < KS; kk++) {
            const int c = 4 * kk + t;
            const double b = (colb < m && c < r) ? A[colb * r + c] : 0.0;
#pragma unroll
            for (int h = 0; h < TT; h++)
                asm volatile(
                    "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                    : "+d"(acc[h][0]), "+d"(acc[h][1])
                    : "d"(la[h][kk]), "d"(b));
        }
#pragma unroll
        for (int h = 0; h < TT; h++)
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int64_t col = 8 * cb + 2 * t + q;
                const int i = 8 * h + g;
                if (col < m && i < r) T[col * r + i] = acc[h][q];
            }
    }
}

// out[e] = sum_b part[b * n + e]: 64 outputs per CTA, 4 threads per output
// each summing every 4th block into 4 accumulators (16 loads in flight), then
// a fixed-order add (deterministic).
__global__ void __launch_bounds__(256) sum_parts_kernel(const double *__restrict__ part, int nblk,
                                                        int n, double *__restrict__ out) {
    __shared__ double red[4][64];
    const int s = threadIdx.x >> 6, o = threadIdx.x & 63;
    for (int e0 = blockIdx.x * 64; e0 < n; e0 += gridDim.x * 64) {
        const int e = e0 + o;
        double a[4] = {0.0, 0.0, 0.0, 0.0};
        if (e < n) {
            int b = s;
            for (; b + 12 < nblk; b += 16) {
#pragma unroll
                for (int j = 0; j < 4; j++) a[j] += part[(int64_t)(b + 4 * j) * n + e];
            }
#pragma unroll
            for (int j = 0; j < 3; j++)
                if (b + 4 * j < nblk) a[j] += part[(int64_t)(b + 4 * j) * n + e];
        }
        red[s][o] = (a[0] + a[1]) + (a[2] + a[3]);
        __syncthreads();
        if (s == 0 && e < n) out[e] = (red[0][o] + red[1][o]) + (red[2][o] + red[3][o]);
        __syncthreads();
    }
}

}  // namespace

void householder_qr(dt_ctx *ctx, const double *A, int64_t m, int64_t n, double *Q, double *R,
                    double *work) {
    DT_CHECK_ARG(m >= n && n > 0, "householder_qr: need m >= n > 0 (m=%lld n=%lld)",
                 (long long)m, (long long)n);
    DT_LAUNCH(ctx, hqr_kernel, 1, LA_NT, 0, A, m, n, Q, R, work);
}

void orth_batch(dt_ctx *ctx, int count, const double *const *A, double *const *Q,
                const int64_t *m, const int64_t *n) {
    int64_t maxm = 0, maxn = 0;
    for (int b = 0; b < count; b++) {
        DT_CHECK_ARG(m[b] >= n[b] && n[b] > 0, "orth_batch: need m >= n > 0");
        maxm = std::max(maxm, m[b]);
        maxn = std::max(maxn, n[b]);
    }
    const int RT = maxn <= 8 ? 8 : (maxn <= 16 ? 16 : 32);
    const int64_t M8 = (maxm + 7) / 8 * 8;
    const size_t smem =
        (2 * (size_t)M8 * (RT + 4) + SM_GP + RT * RT + RT * (RT + 4) + 32) * sizeof(double);
    if (maxn > 32 || smem > 220 * 1024) {
        householder_qr_batch(ctx, count, A, Q, m, n);
        return;
    }
    std::vector<const double *> hA(A, A + count);
    std::vector<double *> hQ(Q, Q + count), hW(count);
    std::vector<int64_t> hm(m, m + count), hn(n, n + count);
    std::vector<DevMem> ws(count);
    for (int b = 0; b < count; b++) {
        ws[b].alloc(ctx, (m[b] * n[b] + n[b]) * sizeof(double));
        hW[b] = ws[b].as<double>();
    }
    DevMem tab(ctx, count * (3 * sizeof(void *) + 2 * sizeof(int64_t)));
    char *base = static_cast<char *>(tab.get());
    const size_t pb = count * sizeof(void *);
    DT_CUDA(cudaMemcpyAsync(base, hA.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + pb, hQ.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + 2 * pb, hW.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + 3 * pb, hm.data(), count * sizeof(int64_t),
                            cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + 3 * pb + count * sizeof(int64_t), hn.data(),
                            count * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    const auto *tA = reinterpret_cast<const double *const *>(base);
    auto *tQ = reinterpret_cast<double *const *>(base + pb);
    auto *tW = reinterpret_cast<double *const *>(base + 2 * pb);
    const auto *tm = reinterpret_cast<const int64_t *>(base + 3 * pb);
    const auto *tn = reinterpret_cast<const int64_t *>(base + 3 * pb + count * sizeof(int64_t));
#define DT_CQR(R)                                                                            \
    do {                                                                                     \
        auto kern = cholqr2_batch_kernel<R>;                                                 \
        smem_limit(ctx, kern, smem);                                                         \
        DT_LAUNCH(ctx, kern, count, SM_NT, smem, tA, tQ, tm, tn, tW);                        \
    } while (0)
    if (RT == 8) DT_CQR(8);
    else if (RT == 16) DT_CQR(16);
    else DT_CQR(32);
#undef DT_CQR
    DT_CUDA(cudaStreamSynchronize(ctx->stream));  // host tables go out of scope
}

void householder_qr_batch(dt_ctx *ctx, int count, const double *const *A, double *const *Q,
                          const int64_t *m, const int64_t *n) {
    // Pointer and size tables plus per-matrix workspaces, staged to the device.
    std::vector<const double *> hA(A, A + count);
    std::vector<double *> hQ(Q, Q + count), hW(count);
    std::vector<int64_t> hm(m, m + count), hn(n, n + count);
    std::vector<DevMem> ws(count);
    for (int b = 0; b < count; b++) {
        DT_CHECK_ARG(m[b] >= n[b] && n[b] > 0, "householder_qr_batch: need m >= n > 0");
        ws[b].alloc(ctx, (m[b] * n[b] + n[b]) * sizeof(double));
        hW[b] = ws[b].as<double>();
    }
    DevMem tab(ctx, count * (3 * sizeof(void *) + 2 * sizeof(int64_t)));
    char *base = static_cast<char *>(tab.get());
    const size_t pb = count * sizeof(void *);
    DT_CUDA(cudaMemcpyAsync(base, hA.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + pb, hQ.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + 2 * pb, hW.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + 3 * pb, hm.data(), count * sizeof(int64_t),
                            cudaMemcpyHostToDevice, ctx->stream));
    DT_CUDA(cudaMemcpyAsync(base + 3 * pb + count * sizeof(int64_t), hn.data(),
                            count * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    DT_LAUNCH(ctx, hqr_batch_kernel, count, 128, 0, reinterpret_cast<const double *const *>(base),
              reinterpret_cast<double *const *>(base + pb),
              reinterpret_cast<const int64_t *>(base + 3 * pb),
              reinterpret_cast<const int64_t *>(base + 3 * pb + count * sizeof(int64_t)),
              reinterpret_cast<double *const *>(base + 2 * pb));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));  // host tables go out of scope
}

void subspace_iter(dt_ctx *ctx, const double *S, int64_t n, double *L, int64_t r, int iters,
                   double *work, int *flag) {
    DT_CHECK_ARG(n >= r && r > 0, "subspace_iter: bad sizes n=%lld r=%lld", (long long)n,
                 (long long)r);
    if (r > 32) {
        DT_LAUNCH(ctx, subspace_wide_kernel, 1, LA_NT, 0, S, n, L, r, iters, work);
        return;
    }
    if (n <= 256) {
        if (r <= 8)
            subspace_mma<8>(ctx, S, (int)n, L, (int)r, iters, work, flag);
        else if (r <= 16)
            subspace_mma<16>(ctx, S, (int)n, L, (int)r, iters, work, flag);
        else
            subspace_mma<32>(ctx, S, (int)n, L, (int)r, iters, work, flag);
        return;
    }
    const size_t base = 2 * r * r * sizeof(double);
    const size_t full_bytes = n * n * sizeof(double);
    const size_t packed_bytes = ((n * (n + 1) / 2 + 1) & ~int64_t(1)) * sizeof(double);
    const size_t zl_bytes = 2 * n * r * sizeof(double);
    const size_t cap = 220 * 1024;
    int s_mode = S_GLOBAL;
    size_t s_bytes = 0;
    if (base + full_bytes + zl_bytes <= cap) {
        s_mode = S_FULL;
        s_bytes = full_bytes;
    } else if (base + packed_bytes + zl_bytes <= cap) {
        s_mode = S_PACKED;
        s_bytes = packed_bytes;
    }
    const int zl_in = base + s_bytes + zl_bytes <= cap;
    const size_t smem = base + s_bytes + (zl_in ? zl_bytes : 0);
    if (r <= 16) {
        smem_limit(ctx, subspace_kernel<16>, smem);
        DT_LAUNCH(ctx, subspace_kernel<16>, 1, LA_NT, smem, S, n, L, r, iters, work, s_mode,
                  zl_in, flag);
    } else {
        smem_limit(ctx, subspace_kernel<32>, smem);
        DT_LAUNCH(ctx, subspace_kernel<32>, 1, LA_NT, smem, S, n, L, r, iters, work, s_mode,
                  zl_in, flag);
    }
}

void lu_inverse(dt_ctx *ctx, const double *A, int64_t n, double *Ainv, double *work,
                int *flag) {
    DT_CHECK_ARG(n > 0 && n <= 8192, "lu_inverse: bad size %lld", (long long)n);
    DT_LAUNCH(ctx, lu_inverse_kernel, 1, LA_NT, n * sizeof(int), A, n, Ainv, work, flag);
}

void orth2_rows(dt_ctx *ctx, double *A, int64_t len1, int64_t len2) {
    // Gram-Schmidt over the rows of A (len1 x len2) equals A = L Q with L the
    // Cholesky factor of A A^T; two passes (CholeskyQR2) for FP64 accuracy.
    DT_CHECK_ARG(len1 > 0 && len1 <= 1024 && len2 >= len1, "orth2: bad sizes %lld x %lld",
                 (long long)len1, (long long)len2);
    DevMem G(ctx, len1 * len1 * sizeof(double));
    DevMem Li(ctx, len1 * len1 * sizeof(double));
    DevMem flag(ctx, sizeof(int));
    DT_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), ctx->stream));
    if (len1 <= 32) {
        const int r = (int)len1;
        const int64_t target = 2LL * ctx->num_sms;
        const int64_t rpb = std::max<int64_t>(256, (len2 + target - 1) / target);
        const int nblk = (int)((len2 + rpb - 1) / rpb);
        DevMem part(ctx, (size_t)nblk * r * r * sizeof(double));
        DevMem T(ctx, (size_t)r * len2 * sizeof(double));
        const unsigned ablocks = std::max(
            1u, std::min<unsigned>(ceil_div(len2 * r, 256), 16u * (unsigned)ctx->num_sms));
        const int RT = r <= 8 ? 8 : (r <= 16 ? 16 : (r <= 24 ? 24 : 32));
        const unsigned mblocks = (unsigned)std::max<int64_t>(
            1, std::min<int64_t>(((len2 + 7) / 8 + 7) / 8, 8LL * ctx->num_sms));
        for (int pass = 0; pass < 2; pass++) {
            const double *src = pass == 0 ? A : T.as<double>();
            double *dst = pass == 0 ? T.as<double>() : A;
#define DT_ROWS(R)                                                                              \
    do {                                                                                        \
        DT_LAUNCH(ctx, rows_gram_mma_kernel<R>, nblk, 256, 0, src, r, len2, rpb,                \
                  part.as<double>());                                                           \
        DT_LAUNCH(ctx, sum_parts_kernel, ceil_div(r * r, 64), 256, 0, part.as<double>(), nblk,    \
                  r * r,                                                                     \
                  G.as<double>());                                                              \
        DT_LAUNCH(ctx, chol_lower_inv_kernel, 1, 256, 2 * r * r * sizeof(double), G.as<double>(), \
                  r, Li.as<double>(), flag.as<int>());                                          \
        DT_LAUNCH(ctx, rows_apply_mma_kernel<R>, mblocks, 256, 0, src, r, len2, Li.as<double>(), \
                  dst);                                                                         \
    } while (0)
            if (RT == 8) DT_ROWS(8);
            else if (RT == 16) DT_ROWS(16);
            else if (RT == 24) DT_ROWS(24);
            else DT_ROWS(32);
#undef DT_ROWS
        }
        int h = 0;
        DT_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h) fail(DT_ERR_NUMERIC, "orth2: rows are linearly dependent");
        return;
    }
    DevMem T(ctx, len1 * len2 * sizeof(double));
    for (int pass = 0; pass < 2; pass++) {
        gemm_f64(ctx, 0, 1, len1, len1, len2, A, len1, A, len1, G.as<double>(), len1, 0.0);
        DT_LAUNCH(ctx, chol_lower_inv_kernel, 1, 256, 2 * len1 * len1 * sizeof(double),
                  G.as<double>(), (int)len1, Li.as<double>(), flag.as<int>());
        gemm_f64(ctx, 0, 0, len1, len2, len1, Li.as<double>(), len1, A, len1, T.as<double>(),
                 len1, 0.0);
        DT_CUDA(cudaMemcpyAsync(A, T.get(), len1 * len2 * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
    }
    int h = 0;
    DT_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h) fail(DT_ERR_NUMERIC, "orth2: rows are linearly dependent");
}

}  // namespace dt
