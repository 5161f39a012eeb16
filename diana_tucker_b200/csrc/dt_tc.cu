// Mixed-precision tensor-core kernels for the dense HOOI hot path (sm_100a):
//
//  * tc_ttm_kernel   Y = X x_n U^T with X in BF16 (hi, or hi+lo), U split into
//                    BF16 hi+lo in shared memory, FP32 accumulation in TMEM.
//                    The mode-n unfolding is never formed: TMA reads X either
//                    K-major (mode 0, contracted index contiguous) or MN-major
//                    (the rows of the output contiguous, 3-D box over
//                    (l, i, b)), and the epilogue writes the result straight
//                    into its destination layout (folded tensor, or the
//                    K-major Y_(n) the Gram consumes).
//  * tc_gram_kernel  split-K S = Y_(n) Y_(n)^T (+ the hi/lo cross term) with
//                    both operands K-major; partial tiles reduced in FP64.
//  * conversions     FP32 -> BF16 hi/lo (+ ||X||^2 in FP64), and the sweep core
//                    G = U^T Y_(N-1) used for the convergence test.
//
// Warp roles in tc_ttm_kernel (192 threads): warp 0 issues TMA, warp 1 owns
// TMEM and issues tcgen05.mma from one thread, warps 2-5 drain TMEM.  Every
// mbarrier wait is bounded (dt_tc.cuh); on timeout the kernel records an error
// and leaves after waiting (bounded) for the copies and MMAs it issued.
#include <cuda.h>

#include <algorithm>
#include <cstring>

#include "dt_tc.cuh"
#include "dt_tc_host.cuh"

namespace dt {
namespace {

using namespace tc;

constexpr int TTM_EPI_WARPS = 8;
constexpr int TTM_THREADS = 64 + 32 * TTM_EPI_WARPS;  // TMA warp, MMA warp, epilogue
constexpr int KC_ELEMS = 64;         // BF16 elements per 128-byte row
constexpr int KC_BYTES = 128 * 128;  // one 128-row x 128-byte K-chunk of A

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
    return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

__device__ __forceinline__ void bf16_split(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// lp, bp and every extent are below 2^31 (tc_ttm_supported): the digits are
// taken with 32-bit divisions, the offset summed in 64 bits.
__device__ __forceinline__ int64_t out_rowbase(const OutMap &om, int64_t lp, int64_t bp) {
    int64_t off = 0;
    uint32_t l = (uint32_t)lp, b = (uint32_t)bp;
    for (int d = 0; d < om.nl; d++) {
        const uint32_t e = (uint32_t)om.dl[d], q = l / e;
        off += (int64_t)(l - q * e) * om.sl[d];
        l = q;
    }
    for (int d = 0; d < om.nb; d++) {
        const uint32_t e = (uint32_t)om.db[d], q = b / e;
        off += (int64_t)(b - q * e) * om.sb[d];
        b = q;
    }
    return off;
}

// ---------------------------------------------------------------------------
// TTM
// ---------------------------------------------------------------------------
template <int JH>
__device__ __forceinline__ void tmem_ld_half(uint32_t taddr, float (&v)[JH]) {
    if constexpr (JH == 8) {
        tmem_ld8(taddr, v);
    } else {
        tmem_ld16(taddr, v);
    }
}

// JP: padded output width (16 or 32); BSPLIT: U as hi + lo (B = [U_hi | U_lo],
// N = 2 JP); ASPLIT: X as hi + lo too (a second MMA X_lo U_hi); FOLDED: the
// output is the folded tensor Y[l, j, b] (else a general OutMap).
template <int JP, bool BSPLIT, bool ASPLIT, bool FOLDED>
__global__ void __launch_bounds__(TTM_THREADS, 1)
    tc_ttm_kernel(const __grid_constant__ CUtensorMap map_hi,
                  const __grid_constant__ CUtensorMap map_lo, const TcTtmArgs a) {
    static_assert(BSPLIT || !ASPLIT, "a split X needs a split U");
    constexpr int NPAD = BSPLIT ? 2 * JP : JP;
    constexpr int JH = JP / 2;  // columns per epilogue warp
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    const int S = a.stages;
    uint8_t *Bt = sm;                                   // kchunks x NPAD rows x 128 B
    const uint32_t b_bytes = (uint32_t)a.kchunks * NPAD * 128;
    uint8_t *Abase = sm + ((b_bytes + 1023) & ~1023u);  // stages
    const uint32_t a_one = (uint32_t)a.kchunks * KC_BYTES;
    const uint32_t stage_bytes = a_one * (ASPLIT ? 2 : 1);
    uint64_t *bars = reinterpret_cast<uint64_t *>(Abase + (size_t)S * stage_bytes);
    uint64_t *full = bars, *empty = bars + S, *tfull = bars + 2 * S, *tempty = bars + 2 * S + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * S + 4);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 1) {
        tmem_alloc(tmem_slot, a.tmem_cols);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&tfull[i], 1);
            mbar_init(&tempty[i], TTM_EPI_WARPS * 32);
        }
        fence_mbar_init();
    }
    // Everything above is private set-up; U and the input tensor may still be
    // in flight from the previous kernel.
    pdl_wait();
    // B = [U_hi | U_lo]^T (split) or U_hi^T, K-major, 128B-swizzled, zero padded.
    // Each U entry is read once (coalesced along k), eight loads in flight per
    // thread, and written as its hi row j and, split, its lo row j + JP.
    {
        const int kmax = a.kchunks * KC_ELEMS;
        const int total = JP * kmax;
        constexpr int UL = 8;
        for (int base = 0; base < total; base += UL * (int)blockDim.x) {
            float v[UL];
#pragma unroll
            for (int u = 0; u < UL; u++) {
                const int e = base + u * (int)blockDim.x + (int)threadIdx.x;
                const int j = e / kmax, k = e - j * kmax;
                v[u] = (e < total && j < a.J && k < a.I)
                           ? (float)a.U[(int64_t)k + (int64_t)a.I * j]
                           : 0.f;
            }
#pragma unroll
            for (int u = 0; u < UL; u++) {
                const int e = base + u * (int)blockDim.x + (int)threadIdx.x;
                if (e < total) {
                    const int j = e / kmax, k = e - j * kmax;
                    __nv_bfloat16 hi, lo;
                    bf16_split(v[u], hi, lo);
                    const int kc = k / KC_ELEMS, kk = k - kc * KC_ELEMS;
                    uint8_t *chunk = Bt + (uint32_t)kc * NPAD * 128;
                    *reinterpret_cast<__nv_bfloat16 *>(chunk + sw128_kmajor_offset(j, kk)) = hi;
                    if (BSPLIT)
                        *reinterpret_cast<__nv_bfloat16 *>(
                            chunk + sw128_kmajor_offset(j + JP, kk)) = lo;
                }
            }
        }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            prefetch_tmap(&map_hi);
            if (ASPLIT) prefetch_tmap(&map_lo);
            int64_t k = 0;
            bool ok = true;
            for (int64_t tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x, k++) {
                const int s = (int)(k % S);
                if (k >= S) ok = mbar_wait(&empty[s], (uint32_t)(((k / S) - 1) & 1), a.err);
                if (!ok) break;
                mbar_expect_tx(&full[s], a.tx_bytes);
                uint8_t *st = Abase + (size_t)s * stage_bytes;
                if (a.kmajor) {
                    const int r0 = (int)(tile * 128);
                    for (int kc = 0; kc < a.kchunks; kc++) {
                        tma_load_2d(st + kc * KC_BYTES, &map_hi, &full[s], kc * KC_ELEMS, r0);
                        if (ASPLIT)
                            tma_load_2d(st + a_one + kc * KC_BYTES, &map_lo, &full[s],
                                        kc * KC_ELEMS, r0);
                    }
                } else {
                    // Each 64-row half of the tile holds its rows for every k
                    // contiguously ([h][k][128 B]); one box covers up to 256
                    // k (fewer, larger boxes stream faster than one per 64 k).
                    const int64_t mb = tile % a.nmb, b = tile / a.nmb;
                    const int l0 = (int)(mb * 128);
                    for (int h = 0; h < 2; h++) {
                        uint8_t *d = st + h * (a_one / 2);
                        for (int kb = 0; kb < a.kboxes; kb++) {
                            const uint32_t off = (uint32_t)kb * a.kbox_rows * 128;
                            tma_load_3d(d + off, &map_hi, &full[s], l0 + h * 64,
                                        kb * a.kbox_rows, (int)b);
                            if (ASPLIT)
                                tma_load_3d(d + a_one + off, &map_lo, &full[s], l0 + h * 64,
                                            kb * a.kbox_rows, (int)b);
                        }
                    }
                }
            }
            // The next kernel may launch once every CTA has issued its last
            // loads.  Triggered at this kernel's start instead, the sweep ran
            // about 0.2 ms slower per decomposition.
            pdl_trigger();
            // Leave no copy in flight: wait (bounded) for every stage issued.
            const int64_t issued = k;
            for (int64_t q = issued - S > 0 ? issued - S : 0; q < issued; q++)
                mbar_wait(&full[q % S], (uint32_t)((q / S) & 1), a.err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t id_full = idesc_bf16(128, NPAD, !a.kmajor, false);
            const uint32_t id_half = idesc_bf16(128, JP, !a.kmajor, false);
            int64_t k = 0;
            bool ok = true;
            for (int64_t tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x, k++) {
                const int s = (int)(k % S);
                const int acc = (int)(k & 1);
                ok = mbar_wait(&full[s], (uint32_t)((k / S) & 1), a.err);
                if (ok && k >= 2) ok = mbar_wait(&tempty[acc], (uint32_t)(((k / 2) - 1) & 1), a.err);
                if (!ok) break;
                tc_fence_after();
                const uint32_t d = tmem_base + (uint32_t)(acc * NPAD);
                const uint32_t st = smem_u32(Abase + (size_t)s * stage_bytes);
                const uint32_t bt = smem_u32(Bt);
                for (int ks = 0; ks < a.ksteps; ks++) {
                    const int kc = ks >> 2, sub = ks & 3;
                    uint64_t ad, adl;
                    if (a.kmajor) {
                        ad = sdesc(st + kc * KC_BYTES + sub * 32, 16, 1024, kSwizzle128B);
                        adl = sdesc(st + a_one + kc * KC_BYTES + sub * 32, 16, 1024, kSwizzle128B);
                    } else {
                        // The second 64 rows of M sit one half-stage (a_one / 2) on.
                        ad = sdesc(st + kc * (KC_BYTES / 2) + sub * 2048, a_one / 2, 1024,
                                   kSwizzle128B);
                        adl = sdesc(st + a_one + kc * (KC_BYTES / 2) + sub * 2048, a_one / 2, 1024,
                                    kSwizzle128B);
                    }
                    const uint64_t bd =
                        sdesc(bt + (uint32_t)kc * NPAD * 128 + sub * 32, 16, 1024, kSwizzle128B);
                    umma_bf16(d, ad, bd, id_full, ks > 0 ? 1u : 0u);
                    if (ASPLIT) umma_bf16(d, adl, bd, id_half, 1u);
                }
                umma_commit(&empty[s]);
                umma_commit(&tfull[acc]);
            }
            // Drain: the last two accumulators' MMAs must finish before dealloc.
            const int64_t issued = k;
            for (int64_t q = issued - 2 > 0 ? issued - 2 : 0; q < issued; q++)
                mbar_wait(&tfull[q & 1], (uint32_t)((q / 2) & 1), a.err);
        }
    } else {
        // Epilogue warps 2..9: two per TMEM lane quarter, each half of the columns.
        const int e = warp - 2;
        const int quarter = warp & 3;
        const int half = e >> 2;
        const int m = quarter * 32 + lane;
        const int j0 = half * JH;
        const int64_t LJ = a.L * a.J;
        int64_t k = 0;
        for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, k++) {
            const int acc = (int)(k & 1);
            if (!mbar_wait(&tfull[acc], (uint32_t)((k / 2) & 1), a.err)) break;
            tc_fence_after();
            const uint32_t taddr =
                tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * NPAD + j0);
            float v[JH];
            tmem_ld_half<JH>(taddr, v);
            if (BSPLIT) {
                float w[JH];
                tmem_ld_half<JH>(taddr + JP, w);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < JH; j++) v[j] += w[j];
            } else {
                tmem_wait_ld();
            }
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
            int64_t lp, bp;
            bool valid;
            if (a.kmajor) {
                lp = 0;
                bp = tile * 128 + m;
                valid = bp < a.B;
            } else {
                const int64_t mb = tile % a.nmb;
                lp = mb * 128 + m;
                bp = tile / a.nmb;
                valid = lp < a.L;
            }
            if (!valid) continue;
            int64_t base, js;
            if (FOLDED) {
                base = lp + bp * LJ;
                js = a.L;
            } else {
                base = out_rowbase(a.om, lp, bp);
                js = a.om.jstride;
            }
            if (a.out_f32) {
#pragma unroll
                for (int j = 0; j < JH; j++)
                    if (j0 + j < a.J) a.out_f32[base + (j0 + j) * js] = v[j];
            } else if (FOLDED && js == 1 && (a.J % JP) == 0) {
                // Contiguous row segment: 16-byte stores.
                __nv_bfloat16 hi[JH], lo[JH];
#pragma unroll
                for (int j = 0; j < JH; j++) bf16_split(v[j], hi[j], lo[j]);
                uint4 *dh = reinterpret_cast<uint4 *>(a.out_hi + base + j0);
#pragma unroll
                for (int q = 0; q < JH / 8; q++) dh[q] = reinterpret_cast<const uint4 *>(hi)[q];
                if (a.out_lo) {
                    uint4 *dl = reinterpret_cast<uint4 *>(a.out_lo + base + j0);
#pragma unroll
                    for (int q = 0; q < JH / 8; q++) dl[q] = reinterpret_cast<const uint4 *>(lo)[q];
                }
            } else {
#pragma unroll
                for (int j = 0; j < JH; j++) {
                    if (j0 + j < a.J) {
                        __nv_bfloat16 hi, lo;
                        bf16_split(v[j], hi, lo);
                        a.out_hi[base + (j0 + j) * js] = hi;
                        if (a.out_lo) a.out_lo[base + (j0 + j) * js] = lo;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, a.tmem_cols);
    }
}

// ---------------------------------------------------------------------------
// Gram: part[z] = Yh Yh^T (and Yh Yl^T in the second half of the columns),
// over this CTA's K-range.  A = rows [0, 128) of the staged Y tile, B = the
// first N rows (Yh rows, then Yl rows, placed back to back).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1)
    tc_gram_kernel(const __grid_constant__ CUtensorMap map_hi,
                   const __grid_constant__ CUtensorMap map_lo, const TcGramArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    const int nck = a.chunks_per_cta;
    const int64_t c0 = (int64_t)blockIdx.x * nck;
    const int64_t c1 = std::min<int64_t>(a.kchunks_total, c0 + nck);
    const int n_my = (int)std::max<int64_t>(0, c1 - c0);
    const uint32_t rows_bytes = (uint32_t)a.Ipad * 128;
    const uint32_t chunk_bytes = a.chunk_bytes;  // >= 128 rows and >= (split ? 2 : 1) * Ipad rows
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + (size_t)nck * chunk_bytes);
    uint64_t *full = bars, *done = bars + nck;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + nck + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        tmem_alloc(tmem_slot, a.tmem_cols);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int c = 0; c < nck; c++) mbar_init(&full[c], 1);
        mbar_init(done, 1);
        fence_mbar_init();
    }
    // Zero the chunk buffers: A reads 128 rows, of which only the first Ipad
    // (or 2*Ipad) are loaded.
    for (uint32_t e = threadIdx.x; e < (uint32_t)nck * chunk_bytes / 16; e += blockDim.x)
        reinterpret_cast<uint4 *>(sm)[e] = make_uint4(0, 0, 0, 0);
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    pdl_wait();  // Y_(n) and the partial buffer are shared with earlier kernels
    bool ok = true;
    if (threadIdx.x == 0) {
        for (int c = 0; c < n_my; c++) {
            mbar_expect_tx(&full[c], a.tx_bytes);
            uint8_t *dst = sm + (size_t)c * chunk_bytes;
            tma_load_2d(dst, &map_hi, &full[c], (int)((c0 + c) * KC_ELEMS), 0);
            if (a.split) tma_load_2d(dst + rows_bytes, &map_lo, &full[c], (int)((c0 + c) * KC_ELEMS), 0);
        }
        const uint32_t idesc = idesc_bf16(128, a.N, false, false);
        for (int c = 0; c < n_my && ok; c++) {
            ok = mbar_wait(&full[c], 0, a.err);
            if (!ok) break;
            tc_fence_after();
            const uint32_t base = smem_u32(sm + (size_t)c * chunk_bytes);
            for (int sub = 0; sub < 4; sub++) {
                const uint64_t ad = sdesc(base + sub * 32, 16, 1024, kSwizzle128B);
                umma_bf16(tmem_base, ad, ad, idesc, (c > 0 || sub > 0) ? 1u : 0u);
            }
        }
        if (ok && n_my > 0) umma_commit(done);
        if (!ok) {
            for (int c = 0; c < n_my; c++) mbar_wait(&full[c], 0, a.err);
        }
    }
    __syncthreads();
    if (n_my > 0 && mbar_wait(done, 0, a.err)) {
        tc_fence_after();
        // Partial tile stored column-major (element (m, g) at g * Ipad + m):
        // lane m of a warp writes consecutive addresses for every column.
        const int m = warp * 32 + lane;
        float *dst = a.part + (int64_t)blockIdx.x * a.Ipad * a.N + m;
        for (int g = 0; g < a.N; g += 16) {
            float v[16];
            tmem_ld16(tmem_base + ((uint32_t)(warp * 32) << 16) + g, v);
            tmem_wait_ld();
            if (m < a.Ipad) {
#pragma unroll
                for (int i = 0; i < 16; i++) dst[(int64_t)(g + i) * a.Ipad] = v[i];
            }
        }
    } else if (n_my == 0) {
        const int m = warp * 32 + lane;
        if (m < a.Ipad)
            for (int g = 0; g < a.N; g++)
                a.part[(int64_t)blockIdx.x * a.Ipad * a.N + (int64_t)g * a.Ipad + m] = 0.f;
    }
    pdl_trigger();  // dependents launch once the partial tile is written
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem_base, a.tmem_cols);
    }
}

// S[i + n*j] = sum_z P_z(i, j) (+ P_z(i, Ipad+j) + P_z(j, Ipad+i)), with the
// partial tiles column-major: P_z(m, g) = part[z][g * Ipad + m].
__global__ void gram_reduce_kernel(const float *__restrict__ part, int nz, int n, int Ipad, int N,
                                   int split, double *__restrict__ S) {
    pdl_wait();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
        const int i = e % n, j = e / n;
        double s = 0.0;
        for (int z = 0; z < nz; z++) {
            const float *p = part + (int64_t)z * Ipad * N;
            s += (double)p[j * Ipad + i];
            if (split) s += (double)p[(Ipad + j) * Ipad + i] + (double)p[(Ipad + i) * Ipad + j];
        }
        S[e] = s;
    }
    pdl_trigger();  // dependents launch once S is written
}

// X (FP32) -> BF16 hi (+ lo) and per-block partial sums of squares (FP64).
__global__ void split_f32_kernel(const float *__restrict__ x, int64_t n,
                                 __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                 double *__restrict__ part) {
    pdl_wait();
    double s = 0.0;
    const int64_t n4 = n / 4;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n4;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float4 v = reinterpret_cast<const float4 *>(x)[e];
        __nv_bfloat16 h[4], l[4];
        bf16_split(v.x, h[0], l[0]);
        bf16_split(v.y, h[1], l[1]);
        bf16_split(v.z, h[2], l[2]);
        bf16_split(v.w, h[3], l[3]);
        reinterpret_cast<uint2 *>(hi)[e] = *reinterpret_cast<uint2 *>(h);
        if (lo) reinterpret_cast<uint2 *>(lo)[e] = *reinterpret_cast<uint2 *>(l);
        s = fma((double)v.x, (double)v.x, s);
        s = fma((double)v.y, (double)v.y, s);
        s = fma((double)v.z, (double)v.z, s);
        s = fma((double)v.w, (double)v.w, s);
    }
    for (int64_t e = n4 * 4 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[e];
        __nv_bfloat16 h, l;
        bf16_split(v, h, l);
        hi[e] = h;
        if (lo) lo[e] = l;
        s = fma((double)v, (double)v, s);
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

// Sweep core from the K-major leaf rows: G[k + K*r] = sum_i Y[i][k] U[i][r]
// in FP64 (hi + lo converts exactly).  A CTA owns 64 columns k; thread
// (c, q) = (t % 64, t / 64) sums the rows i = q, q + 4, ... for all R outputs of
// column k in registers (U staged in shared memory, row-major), and the four
// partial sums are added in a fixed order.  Per-block partial sum of G^2.
template <int RMAX>
__global__ void __launch_bounds__(256) core_rows_kernel(const __nv_bfloat16 *__restrict__ Yh,
                                                        const __nv_bfloat16 *__restrict__ Yl,
                                                        int64_t I, int64_t K,
                                                        const double *__restrict__ U, int R,
                                                        double *__restrict__ G,
                                                        double *__restrict__ part) {
    extern __shared__ double Us[];  // I x RMAX, row i at Us + i * RMAX
    __shared__ double red[4][64];
    __shared__ double s2w[8];
    pdl_wait();
    for (int64_t e = threadIdx.x; e < I * RMAX; e += blockDim.x) {
        const int64_t i = e / RMAX;
        const int r = (int)(e - i * RMAX);
        Us[e] = r < R ? U[i + I * r] : 0.0;
    }
    __syncthreads();
    const int c = threadIdx.x & 63, q = threadIdx.x >> 6;
    const int64_t k = (int64_t)blockIdx.x * 64 + c;
    const bool okk = k < K;
    double acc[RMAX];
#pragma unroll
    for (int r = 0; r < RMAX; r++) acc[r] = 0.0;
    if (okk) {
        for (int64_t i = q; i < I; i += 4) {
            double y = (double)__bfloat162float(Yh[i * K + k]);
            if (Yl) y += (double)__bfloat162float(Yl[i * K + k]);
            const double *u = Us + i * RMAX;
#pragma unroll
            for (int r = 0; r < RMAX; r++) acc[r] = fma(y, u[r], acc[r]);
        }
    }
    pdl_trigger();  // dependents may launch while the core is stored
    double s2 = 0.0;
#pragma unroll
    for (int r = 0; r < RMAX; r++) {
        if (r >= R) break;
        red[q][c] = acc[r];
        __syncthreads();
        if (q == 0 && okk) {
            const double g = (red[0][c] + red[1][c]) + (red[2][c] + red[3][c]);
            G[k + K * r] = g;
            s2 = fma(g, g, s2);
        }
        __syncthreads();
    }
    // s2 lives in the 64 threads of q == 0 (warps 0 and 1).
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_down_sync(0xffffffffu, s2, o);
    if ((threadIdx.x & 31) == 0) s2w[threadIdx.x >> 5] = s2;
    __syncthreads();
    if (threadIdx.x == 0) part[blockIdx.x] = s2w[0] + s2w[1];
}

__global__ void sum_double_kernel(const double *__restrict__ part, int n, double *__restrict__ out) {
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

// ---------------------------------------------------------------------------
// Host side: tensor maps and launchers.
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        DT_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess)
            fail(DT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

CUtensorMap make_map(const void *base, int rank, const uint64_t *dims, const uint64_t *strides_bytes,
                     const uint32_t *box) {
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    cuuint64_t gd[5], gs[4];
    cuuint32_t bx[5], es[5];
    for (int i = 0; i < rank; i++) {
        gd[i] = dims[i];
        bx[i] = box[i];
        es[i] = 1;
    }
    for (int i = 0; i < rank - 1; i++) gs[i] = strides_bytes[i];
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank,
                                   const_cast<void *>(base), gd, gs, bx, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(DT_ERR_CUDA, fmt("cuTensorMapEncodeTiled failed (%d)", (int)r));
    return m;
}

int pad16(int v) { return (v + 15) & ~15; }

}  // namespace

bool tc_ttm_supported(int64_t L, int64_t I, int64_t B, int64_t J) {
    if (J < 1 || J > 32 || I < 1) return false;
    if (I > 64 * 64) return false;  // keeps one stage of A within shared memory
    if (L == 1) return (I % 8) == 0 && B >= 1 && B < (int64_t(1) << 31);
    return L >= 64 && (L % 8) == 0 && L < (int64_t(1) << 31) && B < (int64_t(1) << 31) &&
           I < (int64_t(1) << 31);
}

void tc_ttm(dt_ctx *ctx, const __nv_bfloat16 *Xh, const __nv_bfloat16 *Xl, int64_t L, int64_t I,
            int64_t B, const double *U, int64_t J, const OutMap &om, __nv_bfloat16 *out_hi,
            __nv_bfloat16 *out_lo, float *out_f32, int *err, int usplit) {
    DT_CHECK_ARG(tc_ttm_supported(L, I, B, J), "tc_ttm: unsupported shape L=%lld I=%lld J=%lld",
                 (long long)L, (long long)I, (long long)J);
    TcTtmArgs a{};
    a.kmajor = L == 1;
    a.L = L;
    a.I = I;
    a.B = B;
    a.J = (int)J;
    a.Jpad = pad16((int)J);
    a.split = Xl != nullptr;
    const bool bsplit = usplit < 0 ? a.split : (usplit != 0 || a.split);
    a.Npad = bsplit ? 2 * a.Jpad : a.Jpad;
    a.kchunks = (int)((I + KC_ELEMS - 1) / KC_ELEMS);
    a.ksteps = (int)((I + 15) / 16);
    a.nmb = a.kmajor ? (B + 127) / 128 : (L + 127) / 128;
    a.ntiles = a.kmajor ? a.nmb : a.nmb * B;
    a.U = U;
    a.out_hi = out_hi;
    a.out_lo = out_lo;
    a.out_f32 = out_f32;
    a.om = om;
    a.err = err;
    int cols = 32;
    while (cols < 2 * a.Npad) cols *= 2;
    a.tmem_cols = cols;
    const uint32_t a_one = (uint32_t)a.kchunks * KC_BYTES;
    const uint32_t stage_bytes = a_one * (a.split ? 2 : 1);
    const uint32_t b_bytes = ((uint32_t)a.kchunks * a.Npad * 128 + 1023) & ~1023u;
    const size_t budget = 220 * 1024;
    int S = (int)std::min<size_t>(6, (budget - b_bytes - 1024 - 256) / stage_bytes);
    DT_CHECK_ARG(S >= 2, "tc_ttm: contraction length %lld too large for shared memory", (long long)I);
    a.stages = S;
    // Bytes the TMA delivers per stage (boxes are counted whole, OOB included).
    a.tx_bytes = stage_bytes;
    CUtensorMap mh, ml;
    if (a.kmajor) {
        const uint64_t dims[2] = {(uint64_t)I, (uint64_t)B};
        const uint64_t str[1] = {(uint64_t)I * 2};
        const uint32_t box[2] = {KC_ELEMS, 128};
        mh = make_map(Xh, 2, dims, str, box);
        ml = Xl ? make_map(Xl, 2, dims, str, box) : mh;
    } else {
        const uint64_t dims[3] = {(uint64_t)L, (uint64_t)I, (uint64_t)B};
        const uint64_t str[2] = {(uint64_t)L * 2, (uint64_t)L * I * 2};
        // One box per half-tile over all k when the contraction is at most
        // 256 long, else one per 64-element chunk.
        a.kbox_rows = a.kchunks <= 4 ? a.kchunks * KC_ELEMS : KC_ELEMS;
        a.kboxes = a.kchunks * KC_ELEMS / a.kbox_rows;
        const uint32_t box[3] = {64, (uint32_t)a.kbox_rows, 1};
        mh = make_map(Xh, 3, dims, str, box);
        ml = Xl ? make_map(Xl, 3, dims, str, box) : mh;
    }
    const size_t smem = 1024 + b_bytes + (size_t)S * stage_bytes + (2 * S + 4) * 8 + 16;
    const unsigned grid = (unsigned)std::min<int64_t>(a.ntiles, ctx->num_sms);
    const bool folded = om.nl == 1 && om.nb == 1 && om.dl[0] == std::max<int64_t>(L, 1) &&
                        om.sl[0] == 1 && om.sb[0] == L * J && om.jstride == L;
    auto go = [&](auto kernel) {
        smem_limit(ctx, kernel, smem);
        DT_LAUNCH_PDL(ctx, kernel, grid, TTM_THREADS, smem, mh, ml, a);
    };
#define DT_TTM_GO(JP)                                                                    \
    do {                                                                                 \
        if (a.split)                                                                     \
            folded ? go(tc_ttm_kernel<JP, true, true, true>)                             \
                   : go(tc_ttm_kernel<JP, true, true, false>);                           \
        else if (bsplit)                                                                 \
            folded ? go(tc_ttm_kernel<JP, true, false, true>)                            \
                   : go(tc_ttm_kernel<JP, true, false, false>);                          \
        else                                                                             \
            folded ? go(tc_ttm_kernel<JP, false, false, true>)                           \
                   : go(tc_ttm_kernel<JP, false, false, false>);                         \
    } while (0)
    if (a.Jpad == 16)
        DT_TTM_GO(16);
    else
        DT_TTM_GO(32);
#undef DT_TTM_GO
}

bool tc_gram_supported(int64_t I, int64_t K) {
    return I >= 1 && I <= 128 && (K % 8) == 0 && K >= 1 && K < (int64_t(1) << 31);
}

namespace {

// The split-K layout of tc_gram: partial tiles nz x Ipad x N, nck chunks each.
void gram_layout(int64_t I, int64_t K, bool split, TcGramArgs &a, int64_t &nz) {
    a.split = split;
    a.Ipad = (int)((I + 7) & ~int64_t(7));
    a.N = pad16(a.split ? 2 * a.Ipad : a.Ipad);
    a.kchunks_total = (K + KC_ELEMS - 1) / KC_ELEMS;
    // At most 16 partial tiles: the MMA work is small, the FP64 reduction of
    // the partials is what grows with the split.
    const int64_t target = 16;
    int nck = (int)std::max<int64_t>(1, (a.kchunks_total + target - 1) / target);
    a.chunk_bytes = (uint32_t)std::max<int64_t>(KC_BYTES, (a.split ? 2 : 1) * a.Ipad * 128);
    a.chunk_bytes = (a.chunk_bytes + 1023) & ~1023u;
    while (nck > 1 && (size_t)nck * a.chunk_bytes > 200 * 1024) nck--;
    nz = (a.kchunks_total + nck - 1) / nck;
    a.chunks_per_cta = nck;
}

}  // namespace

size_t tc_gram_scratch_bytes(int64_t I, int64_t K, bool split) {
    TcGramArgs a{};
    int64_t nz = 0;
    gram_layout(I, K, split, a, nz);
    return (size_t)nz * a.Ipad * a.N * sizeof(float);
}

void tc_gram(dt_ctx *ctx, const __nv_bfloat16 *Yh, const __nv_bfloat16 *Yl, int64_t I, int64_t K,
             double *S, int *err, void *scratch) {
    DT_CHECK_ARG(tc_gram_supported(I, K), "tc_gram: unsupported I=%lld K=%lld", (long long)I,
                 (long long)K);
    TcGramArgs a{};
    int64_t nz = 0;
    gram_layout(I, K, Yl != nullptr, a, nz);
    const int nck = a.chunks_per_cta;
    a.tx_bytes = (uint32_t)((a.split ? 2 : 1) * a.Ipad * 128);
    int cols = 32;
    while (cols < a.N) cols *= 2;
    a.tmem_cols = cols;
    a.err = err;
    DevMem part;
    if (!scratch) part.alloc(ctx, (size_t)nz * a.Ipad * a.N * sizeof(float));
    a.part = scratch ? static_cast<float *>(scratch) : part.as<float>();
    const uint64_t dims[2] = {(uint64_t)K, (uint64_t)I};
    const uint64_t str[1] = {(uint64_t)K * 2};
    const uint32_t box[2] = {KC_ELEMS, (uint32_t)a.Ipad};
    CUtensorMap mh = make_map(Yh, 2, dims, str, box);
    CUtensorMap ml = Yl ? make_map(Yl, 2, dims, str, box) : mh;
    const size_t smem = 1024 + (size_t)nck * a.chunk_bytes + (nck + 2) * 8 + 16;
    smem_limit(ctx, tc_gram_kernel, smem);
    DT_LAUNCH_PDL(ctx, tc_gram_kernel, (unsigned)nz, 128, smem, mh, ml, a);
    const int n = (int)I;
    DT_LAUNCH_PDL(ctx, gram_reduce_kernel, std::max(1u, ceil_div((int64_t)n * n, 256)), 256, 0,
              a.part, (int)nz, n, a.Ipad, a.N, a.split, S);
}

void split_f32(dt_ctx *ctx, const float *x, int64_t n, __nv_bfloat16 *hi, __nv_bfloat16 *lo,
               double *sumsq_out) {
    const int blocks = std::max(1, std::min<int>(4 * ctx->num_sms, (int)ceil_div(n / 4 + 1, 256)));
    DevMem part(ctx, (size_t)blocks * sizeof(double));
    DT_LAUNCH_PDL(ctx, split_f32_kernel, blocks, 256, 0, x, n, hi, lo, part.as<double>());
    DT_LAUNCH_PDL(ctx, sum_double_kernel, 1, 1024, 0, part.as<double>(), blocks, sumsq_out);
}

void split_f32_chunks(dt_ctx *ctx, const ChunkedUpload &up, __nv_bfloat16 *hi,
                      __nv_bfloat16 *lo, double *sumsq_out) {
    const float *dx = up.dst.as<float>();
    const int bpc =
        std::max(1, std::min<int>(2 * ctx->num_sms, (int)ceil_div(up.step / 4 + 1, 256)));
    DevMem part(ctx, (size_t)up.chunks * bpc * sizeof(double));
    for (int c = 0; c < up.chunks; c++) {
        up.wait(ctx, c);
        const int64_t off = up.offset(c);
        DT_LAUNCH_PDL(ctx, split_f32_kernel, bpc, 256, 0, dx + off, up.length(c), hi + off,
                  lo ? lo + off : nullptr, part.as<double>() + (size_t)c * bpc);
    }
    // Partials in chunk order: the same sum on every call.
    DT_LAUNCH_PDL(ctx, sum_double_kernel, 1, 1024, 0, part.as<double>(), up.chunks * bpc, sumsq_out);
}

size_t core_rows_scratch_bytes(int64_t K) {
    return (size_t)std::max<int64_t>(1, ceil_div(K, 64)) * sizeof(double);
}

void core_rows(dt_ctx *ctx, const __nv_bfloat16 *Yh, const __nv_bfloat16 *Yl, int64_t I, int64_t K,
               const double *U, int64_t R, double *G, double *g2_out, void *scratch) {
    DT_CHECK_ARG(R <= 32, "core_rows: R %lld > 32", (long long)R);
    const int blocks = (int)std::max<int64_t>(1, ceil_div(K, 64));
    DevMem own;
    if (!scratch) own.alloc(ctx, (size_t)blocks * sizeof(double));
    double *part = scratch ? static_cast<double *>(scratch) : own.as<double>();
#define DT_CORE_ROWS(RM)                                                                     \
    do {                                                                                     \
        const size_t smem = (size_t)I * RM * sizeof(double);                                 \
        smem_limit(ctx, core_rows_kernel<RM>, smem);                                         \
        DT_LAUNCH_PDL(ctx, core_rows_kernel<RM>, blocks, 256, smem, Yh, Yl, I, K, U, (int)R, G,  \
                  part);                                                                     \
    } while (0)
    if (R <= 8)
        DT_CORE_ROWS(8);
    else if (R <= 16)
        DT_CORE_ROWS(16);
    else
        DT_CORE_ROWS(32);
#undef DT_CORE_ROWS
    DT_LAUNCH_PDL(ctx, sum_double_kernel, 1, 1024, 0, part, blocks, g2_out);
}

}  // namespace dt
