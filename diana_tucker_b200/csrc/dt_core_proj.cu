// The final FP64 core projection of the mixed-precision HOOI, first step:
//
//     T[r0, r1, s] = sum_{i0, i1} U0[i0, r0] X[i0, i1, s] U1[i1, r1]
//
// over the slices s of X (every mode but the two lowest), straight from the
// FP32 X and in FP64 arithmetic on the FP64 tensor cores (mma.sync m8n8k4).
// X is read once and the only intermediate written is T (R0 R1 prod_{m>=2}
// I_m doubles, 19 MB for 96^4 at rank 16), where contracting mode by mode
// would write and re-read X x_m U_m^T (96^3 x 16 doubles, 113 MB) in FP64.
// The remaining modes of T are contracted by the dense TTM kernels.
//
// One persistent CTA per SM, eight warps; per slice:
//  * the slice (I0 x I1 floats) arrives by 16-byte cp.async into one of two
//    shared-memory stages while the previous slice is computed; columns are
//    padded to a pitch = 4 mod 32 floats so the B-fragment loads (k = t,
//    column g) hit 32 distinct banks;
//  * W = U0^T X_s (RM x I1) in FP64: warps take 8 x 8 output tiles, the
//    k-loop runs over i0; W goes to shared memory (pitch = 4 mod 16 doubles);
//  * T_s = W U1 (RM x RM): one 8 x 8 tile per warp, k over i1;
//  * rows/columns beyond R0/R1 and k beyond I0/I1 are zero padding.
#include <algorithm>

#include "dt_kernels.cuh"

namespace dt {
namespace {

constexpr int CP_THREADS = 256;
constexpr int CP_MAXT = 16;  // W tiles per warp: (RM / 8) x ceil(I1 / 8) / 8

__device__ __forceinline__ void cpa16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cpa4(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// volatile: the compiler must not execute a guarded MMA unconditionally.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

struct CoreSliceArgs {
    const float *X;
    int I0, I1;
    int64_t S;
    const double *U0, *U1;  // I0 x R0, I1 x R1 col-major
    int R0, R1;
    double *T;              // R0 x R1 x S col-major
    int xp;                 // slice column pitch (floats), = 4 mod 32
    int k0, k1;             // I0, I1 rounded up to 4
    int up;                 // pitch of U0t / U1t / W (doubles), = 4 mod 16
    int vec16;              // 16-byte copies (I0 % 4 == 0 and X 16-byte aligned)
};

template <int RM>
__global__ void __launch_bounds__(CP_THREADS, 1) core_slices_kernel(const CoreSliceArgs a) {
    extern __shared__ __align__(16) uint8_t cp_smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    double *U0t = reinterpret_cast<double *>(cp_smem);  // RM rows x up: U0t[r][i0]
    double *U1t = U0t + RM * a.up;                       // RM rows x up: U1t[r][i1]
    double *W = U1t + RM * a.up;                         // RM rows x up: W[r][i1]
    float *Xs = reinterpret_cast<float *>(W + RM * a.up);  // 2 stages x I1 columns x xp
    const int stage_floats = a.I1 * a.xp;
    pdl_trigger();
    // Zero the padding that the fragments read (k beyond I0 / I1, rows beyond R).
    for (int e = threadIdx.x; e < 3 * RM * a.up; e += CP_THREADS) U0t[e] = 0.0;
    for (int e = threadIdx.x; e < 2 * stage_floats; e += CP_THREADS) Xs[e] = 0.f;
    __syncthreads();
    pdl_wait();
    for (int e = threadIdx.x; e < a.I0 * a.R0; e += CP_THREADS) {
        const int i = e % a.I0, r = e / a.I0;
        U0t[r * a.up + i] = a.U0[e];
    }
    for (int e = threadIdx.x; e < a.I1 * a.R1; e += CP_THREADS) {
        const int i = e % a.I1, r = e / a.I1;
        U1t[r * a.up + i] = a.U1[e];
    }
    const int64_t slice_elems = (int64_t)a.I0 * a.I1;
    auto issue = [&](int64_t s, int st) {
        float *dst = Xs + st * stage_floats;
        const float *src = a.X + s * slice_elems;
        if (a.vec16) {
            const int per_col = a.I0 / 4;
            for (int e = threadIdx.x; e < a.I1 * per_col; e += CP_THREADS) {
                const int c = e / per_col, q = e - c * per_col;
                cpa16(dst + c * a.xp + 4 * q, src + (int64_t)c * a.I0 + 4 * q);
            }
        } else {
            for (int e = threadIdx.x; e < a.I1 * a.I0; e += CP_THREADS) {
                const int c = e / a.I0, i = e - c * a.I0;
                cpa4(dst + c * a.xp + i, src + (int64_t)c * a.I0 + i);
            }
        }
        cpa_commit();
    };
    const int mt_w = RM / 8, nt_w = (a.I1 + 7) / 8;
    int64_t s = blockIdx.x;
    if (s < a.S) issue(s, 0);
    for (int it = 0; s < a.S; s += gridDim.x, it++) {
        const int st = it & 1;
        const int64_t sn = s + gridDim.x;
        if (sn < a.S) {
            issue(sn, st ^ 1);
            cpa_wait<1>();
        } else {
            cpa_wait<0>();
        }
        __syncthreads();
        const float *Xc = Xs + st * stage_floats;
        // W = U0^T X_s: tiles (mt over r0, nt over i1), k over i0.  Warp w
        // owns tiles w, w + 8, ...; their k-loops run interleaved.
        {
            const double *arow[CP_MAXT];
            const float *bcol[CP_MAXT];
            double d0[CP_MAXT], d1[CP_MAXT];
            int ntl = 0;
#pragma unroll
            for (int q = 0; q < CP_MAXT; q++) {
                const int tile = w + 8 * q;
                const bool on = tile < mt_w * nt_w;
                const int mt = on ? tile % mt_w : 0, nt = on ? tile / mt_w : 0;
                arow[q] = U0t + (8 * mt + g) * a.up + t;
                bcol[q] = Xc + min(8 * nt + g, a.I1 - 1) * a.xp + t;  // columns past I1 discarded
                d0[q] = d1[q] = 0.0;
                ntl += on;
            }
            for (int k = 0; k < a.k0; k += 4) {
#pragma unroll
                for (int q = 0; q < CP_MAXT; q++)
                    if (q < ntl) dmma(d0[q], d1[q], arow[q][k], (double)bcol[q][k]);
            }
#pragma unroll
            for (int q = 0; q < CP_MAXT; q++) {
                if (q >= ntl) break;
                const int tile = w + 8 * q, mt = tile % mt_w, nt = tile / mt_w;
                const int c0 = 8 * nt + 2 * t;
                if (c0 < a.I1) W[(8 * mt + g) * a.up + c0] = d0[q];
                if (c0 + 1 < a.I1) W[(8 * mt + g) * a.up + c0 + 1] = d1[q];
            }
        }
        __syncthreads();
        // T_s = W U1: tiles (mt over r0, nt over r1), k over i1, two
        // accumulator pairs per tile (even / odd k-steps).
        for (int tile = w; tile < mt_w * mt_w; tile += CP_THREADS / 32) {
            const int mt = tile % mt_w, nt = tile / mt_w;
            const double *arow = W + (8 * mt + g) * a.up + t;
            const double *brow = U1t + (8 * nt + g) * a.up + t;
            double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
            int k = 0;
            for (; k + 8 <= a.k1; k += 8) {
                dmma(d0, d1, arow[k], brow[k]);
                dmma(e0, e1, arow[k + 4], brow[k + 4]);
            }
            for (; k < a.k1; k += 4) dmma(d0, d1, arow[k], brow[k]);
            d0 += e0;
            d1 += e1;
            const int r0 = 8 * mt + g, r1 = 8 * nt + 2 * t;
            double *out = a.T + s * a.R0 * a.R1;
            if (r0 < a.R0) {
                if (r1 < a.R1) out[r0 + (int64_t)a.R0 * r1] = d0;
                if (r1 + 1 < a.R1) out[r0 + (int64_t)a.R0 * (r1 + 1)] = d1;
            }
        }
        __syncthreads();  // stage st and W are reused by the next slices
    }
}

constexpr int up_pitch(int k) { return k + ((4 - k % 16) + 16) % 16; }
constexpr int xs_pitch(int k) { return k + ((4 - k % 32) + 32) % 32; }

size_t core_slices_smem(int64_t I0, int64_t I1, int RM) {
    const int k0 = (int)((I0 + 3) & ~int64_t(3)), k1 = (int)((I1 + 3) & ~int64_t(3));
    const int up = up_pitch(std::max(k0, k1));
    const int xp = xs_pitch(k0);
    return (size_t)3 * RM * up * sizeof(double) + (size_t)2 * I1 * xp * sizeof(float);
}

}  // namespace

bool core_slices_supported(int64_t I0, int64_t I1, int64_t R0, int64_t R1) {
    if (I0 < 1 || I1 < 1 || R0 < 1 || R1 < 1 || R0 > 32 || R1 > 32 || R0 > I0 || R1 > I1)
        return false;
    const int RM = (int)std::max<int64_t>(8, ((std::max(R0, R1) + 7) / 8) * 8);
    // W tiles per warp within CP_MAXT.
    if ((RM / 8) * ((I1 + 7) / 8) > 8 * CP_MAXT) return false;
    return I0 <= 1024 && I1 <= 1024 && core_slices_smem(I0, I1, RM) <= 200 * 1024;
}

void core_slices_f64(dt_ctx *ctx, const float *X, int64_t I0, int64_t I1, int64_t S,
                     const double *U0, int64_t R0, const double *U1, int64_t R1, double *T) {
    DT_CHECK_ARG(core_slices_supported(I0, I1, R0, R1), "core_slices_f64: unsupported shape");
    CoreSliceArgs a{};
    a.X = X;
    a.I0 = (int)I0;
    a.I1 = (int)I1;
    a.S = S;
    a.U0 = U0;
    a.U1 = U1;
    a.R0 = (int)R0;
    a.R1 = (int)R1;
    a.T = T;
    a.k0 = (int)((I0 + 3) & ~int64_t(3));
    a.k1 = (int)((I1 + 3) & ~int64_t(3));
    a.up = up_pitch(std::max(a.k0, a.k1));
    a.xp = xs_pitch(a.k0);
    a.vec16 = (I0 % 4 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    const int RM = (int)std::max<int64_t>(8, ((std::max(R0, R1) + 7) / 8) * 8);
    const size_t smem = core_slices_smem(I0, I1, RM);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(S, ctx->num_sms));
    auto go = [&](auto kernel) {
        smem_limit(ctx, kernel, smem);
        DT_LAUNCH_PDL(ctx, kernel, grid, CP_THREADS, smem, a);
    };
    if (RM == 8)
        go(core_slices_kernel<8>);
    else if (RM == 16)
        go(core_slices_kernel<16>);
    else if (RM == 24)
        go(core_slices_kernel<24>);
    else
        go(core_slices_kernel<32>);
}

}  // namespace dt
