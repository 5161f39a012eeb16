// Small dense FP64 linear algebra on the GPU: the reference's LAPACK calls
// (src/operator/operator_double.cpp:84-155) and its ALS_ leading-subspace step
// (template/algorithm/tucker/hooi_als.tpp:7-34), kept on the device so a HOOI
// sweep never round-trips to the host.  These matrices are tiny (R x R, I_n x R,
// I_n x I_n): one CTA per problem, latency-bound, so the code minimises block
// barriers rather than flops.
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
// one warp, then Rinv = R^{-1} (upper, row-major).  Returns false on a
// non-positive pivot.  Runs in warp 0 only.
__device__ bool warp_chol_inv(double *G, double *Rinv, int r) {
    const int lane = threadIdx.x & 31;
    bool ok = true;
    const double g00 = G[0];
    for (int k = 0; k < r; k++) {
        const double d = G[k * r + k];
        if (!(d > 1e-28 * g00)) ok = false;
        const double rkk = sqrt(fmax(d, 1e-300));
        __syncwarp();
        for (int c = k + 1 + lane; c < r; c += 32) G[k * r + c] /= rkk;
        __syncwarp();
        if (lane == 0) G[k * r + k] = rkk;
        for (int i = k + 1; i < r; i++) {
            const double rki = G[k * r + i];
            for (int c = i + lane; c < r; c += 32) G[i * r + c] = fma(-rki, G[k * r + c], G[i * r + c]);
        }
        __syncwarp();
    }
    // Column c of R^{-1}: back substitution, one lane per column.
    for (int c = lane; c < r; c += 32) {
        for (int i = 0; i < r; i++) Rinv[i * r + c] = 0.0;
        Rinv[c * r + c] = 1.0 / G[c * r + c];
        for (int i = c - 1; i >= 0; i--) {
            double s = 0.0;
            for (int j = i + 1; j <= c; j++) s = fma(G[i * r + j], Rinv[j * r + c], s);
            Rinv[i * r + c] = -s / G[i * r + i];
        }
    }
    __syncwarp();
    return ok;
}

// Subspace iteration L <- orth(S L), `iters` times, one CTA.  S (n x n,
// symmetric), L and Z (n x r) live in shared memory when they fit, else in
// the global workspace.  Each step orthonormalises with CholeskyQR2; a
// Cholesky breakdown (rank-deficient S L) switches that step to Householder.
__global__ void __launch_bounds__(LA_NT) subspace_kernel(const double *Sg, int64_t n,
                                                         double *Lg, int64_t r, int iters,
                                                         double *work, int s_in_smem,
                                                         int zl_in_smem, int *flag) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[33];
    __shared__ int bad;
    const int t = threadIdx.x;
    double *G = sm;                // r*r
    double *Ri = sm + r * r;       // r*r
    double *cur = sm + 2 * r * r;  // after the two r x r blocks
    const double *S = Sg;
    if (s_in_smem) {
        double *Ss = cur;
        for (int64_t e = t; e < n * n; e += blockDim.x) Ss[e] = Sg[e];
        S = Ss;
        cur += n * n;
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
    for (int it = 0; it < iters; it++) {
        // Z = S L
        for (int64_t e = t; e < n * r; e += blockDim.x) {
            const int64_t i = e % n, c = e / n;
            const double *lc = L + c * n;
            double s = 0.0;
            for (int64_t k = 0; k < n; k++) s = fma(S[i + n * k], lc[k], s);
            Z[e] = s;
        }
        __syncthreads();
        // Two CholeskyQR passes: Z -> L -> Z, final basis copied to L.
        bool broke = false;
        for (int pass = 0; pass < 2 && !broke; pass++) {
            double *src = pass == 0 ? Z : L;
            double *dst = pass == 0 ? L : Z;
            for (int e = t; e < r * r; e += blockDim.x) {
                const int a = e / (int)r, b = e % (int)r;
                if (b < a) continue;
                const double *ca = src + (int64_t)a * n, *cb = src + (int64_t)b * n;
                double s = 0.0;
                for (int64_t k = 0; k < n; k++) s = fma(ca[k], cb[k], s);
                G[a * r + b] = s;
                G[b * r + a] = s;
            }
            __syncthreads();
            if (t < 32) {
                const bool ok = warp_chol_inv(G, Ri, (int)r);
                if (t == 0) bad = ok ? 0 : 1;
            }
            __syncthreads();
            if (bad) {
                broke = true;
                break;
            }
            for (int64_t e = t; e < n * r; e += blockDim.x) {
                const int64_t i = e % n, c = e / n;
                double s = 0.0;
                for (int64_t k = 0; k <= c; k++) s = fma(src[i + k * n], Ri[k * r + c], s);
                dst[e] = s;
            }
            __syncthreads();
        }
        if (broke) {
            // Householder on S L (still in Z when the first pass broke, in L
            // when the second did): copy into the workspace and rebuild L.
            const double *srcz = Z;
            for (int64_t e = t; e < n * r; e += blockDim.x) hwork[e] = srcz[e];
            __syncthreads();
            hqr_device(hwork, n, r, hwork + n * r, L, red);
            if (t == 0 && flag) atomicOr(flag, 2);
            __syncthreads();
        } else {
            for (int64_t e = t; e < n * r; e += blockDim.x) L[e] = Z[e];
            __syncthreads();
        }
    }
    for (int64_t e = t; e < n * r; e += blockDim.x) Lg[e] = L[e];
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

// Cholesky of the r x r SPD G (col-major) and L^{-1} (lower) for the row
// orthonormalisation; one CTA, r small.  Output Linv col-major.
__global__ void chol_lower_inv_kernel(const double *Gg, int r, double *Linv, int *flag) {
    extern __shared__ double sm[];
    double *G = sm, *Ri = sm + r * r;
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) G[e] = Gg[e];  // symmetric
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool ok = warp_chol_inv(G, Ri, r);
        if (!ok && threadIdx.x == 0) atomicOr(flag, 1);
    }
    __syncthreads();
    // G = R^T R with R upper; L = R^T, so L^{-1} = (R^{-1})^T.
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int i = e % r, c = e / r;  // Linv(i, c) = Rinv(c, i)
        Linv[e] = Ri[c * r + i];
    }
}

}  // namespace

void householder_qr(dt_ctx *ctx, const double *A, int64_t m, int64_t n, double *Q, double *R,
                    double *work) {
    DT_CHECK_ARG(m >= n && n > 0, "householder_qr: need m >= n > 0 (m=%lld n=%lld)",
                 (long long)m, (long long)n);
    DT_LAUNCH(ctx, hqr_kernel, 1, LA_NT, 0, A, m, n, Q, R, work);
}

void subspace_iter(dt_ctx *ctx, const double *S, int64_t n, double *L, int64_t r, int iters,
                   double *work, int *flag) {
    DT_CHECK_ARG(n >= r && r > 0 && r <= 1024, "subspace_iter: bad sizes n=%lld r=%lld",
                 (long long)n, (long long)r);
    const size_t base = 2 * r * r * sizeof(double);
    const size_t s_bytes = n * n * sizeof(double);
    const size_t zl_bytes = 2 * n * r * sizeof(double);
    const size_t cap = 200 * 1024;
    int s_in = base + s_bytes + zl_bytes <= cap;
    int zl_in = base + (s_in ? s_bytes : 0) + zl_bytes <= cap;
    const size_t smem = base + (s_in ? s_bytes : 0) + (zl_in ? zl_bytes : 0);
    DT_CUDA(cudaFuncSetAttribute(subspace_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    DT_LAUNCH(ctx, subspace_kernel, 1, LA_NT, smem, S, n, L, r, iters, work, s_in, zl_in, flag);
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
    DevMem T(ctx, len1 * len2 * sizeof(double));
    DevMem flag(ctx, sizeof(int));
    DT_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), ctx->stream));
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
