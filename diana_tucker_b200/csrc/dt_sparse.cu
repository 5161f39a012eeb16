// Sparse Tucker hot path: SpTensor construction with one mode-sorted copy of
// the nonzeros per mode, the TTMc (row-wise Kronecker accumulation of
// template/function/sp_tensor.tpp:288-417), its two contractions ttmc_mTR /
// ttmc_mTL (sp_tensor.tpp:236-365), and the sparse HOOI power sweep
// (template/algorithm/sp_tucker/sp_hooi_als.tpp:48-118).
//
// TTMc work decomposition: the nonzeros of every non-empty mode-n row are cut
// into chunks of at most CHUNK nonzeros; one warp owns one chunk and keeps the
// row's P = prod_{m != n} R_m accumulators in registers (P/32 per lane).  A row
// that fits one chunk is written directly; a longer row (Zipf-skewed heads)
// writes per-chunk partial rows that a second kernel sums in chunk order.  The
// output is therefore deterministic and needs no floating-point atomics.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dt_kernels.cuh"

namespace dt {
namespace {

constexpr int MAXD = 8;
constexpr int64_t CHUNK = 512;
constexpr int64_t TASK_PACK = 512;
constexpr int64_t TASK_PIECE = 2048;

struct ModeCopy {
    // Nonzeros sorted by this mode's index.
    DevMem other;       // int32 [ndim-1][nnz]: the other modes' indices, in mode order
    DevMem val;         // double [nnz]
    int64_t nrows = 0;  // non-empty rows
    DevMem rows;        // int32 [nrows]: row id of compact row k
    DevMem rowptr;      // int64 [nrows+1]
    int64_t nchunks = 0;
    DevMem chunk_row;   // int32 [nchunks]: compact row of the chunk
    DevMem chunk_beg;   // int64 [nchunks]
    DevMem chunk_slot;  // int32 [nchunks]: -1 = write row directly, else partial slot
    int64_t nslots = 0;
    int64_t nmulti = 0;   // rows with more than one chunk
    DevMem multi_row;     // int32 [nmulti]: compact row
    DevMem multi_first;   // int32 [nmulti]: first partial slot
    DevMem multi_count;   // int32 [nmulti]
    // Task list of the 3-way TTMc kernel: runs of whole consecutive rows with
    // at most TASK_PACK nonzeros in all, and pieces of at most TASK_PIECE
    // nonzeros of longer rows; sorted by size, largest first.
    int64_t ntasks = 0;
    DevMem task_beg;      // int64 [ntasks]
    DevMem task_end;      // int64 [ntasks]
    DevMem task_row;      // int32 [ntasks]: compact row of the first nonzero
    DevMem task_slot;     // int32 [ntasks]: -1 = rows written directly, else partial slot
    int64_t tslots = 0;
    int64_t tmulti = 0;   // rows cut into several pieces
    DevMem tmulti_row, tmulti_first, tmulti_count;
};

struct FactorSet {
    const double *U[MAXD];  // transposed factors: row i of mode m at U[m] + i*R[m]
    int R[MAXD];
};

}  // namespace
}  // namespace dt

struct dt_sptensor {
    dt_ctx *ctx = nullptr;
    int ndim = 0;
    int64_t nnz = 0;
    int64_t shape[dt::MAXD] = {};
    double fnorm = 0.0;
    std::vector<dt::ModeCopy> modes;
};

namespace dt {
namespace {

__global__ void narrow_index_kernel(const int64_t *__restrict__ in, int64_t n, int64_t bound,
                                    int32_t *__restrict__ out, int *__restrict__ bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = in[e];
        if (v < 0 || v >= bound) {
            atomicOr(bad, 1);
            out[e] = 0;
        } else {
            out[e] = (int32_t)v;
        }
    }
}

__global__ void iota_kernel(int32_t *__restrict__ a, int64_t n) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        a[e] = (int32_t)e;
}

template <class T>
__global__ void gather_kernel(const T *__restrict__ src, const int32_t *__restrict__ perm,
                              int64_t n, T *__restrict__ dst) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        dst[e] = src[perm[e]];
}

// ---------------------------------------------------------------------------
// TTMc row kernel.  One warp per chunk.  Lane l owns Kronecker entries
// p = l + 32 q (q < PL).  For 3-way tensors with R_a | 32 the entry p =
// pa + R_a pb maps to a lane-constant pa, so each nonzero costs one factor-row
// load per mode, PL shuffles and PL FMAs per lane.
// ---------------------------------------------------------------------------
template <int PL, bool FAST3>
__global__ void __launch_bounds__(256) ttmc_rows_kernel(
    const int32_t *__restrict__ other, const double *__restrict__ val, int64_t nnz, int nother,
    const int64_t *__restrict__ rowptr, const int32_t *__restrict__ chunk_row,
    const int64_t *__restrict__ chunk_beg, const int32_t *__restrict__ chunk_slot,
    int64_t nchunks, FactorSet f, int P, double *__restrict__ Yc, double *__restrict__ Ypart) {
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // Per-lane Kronecker coordinates (FAST3: p = pa + Ra*pb).
    const int Ra = f.R[0];
    const int pa = FAST3 ? (lane % Ra) : 0;
    const int pb0 = FAST3 ? (lane / Ra) : 0;
    const int pbstep = FAST3 ? (32 / Ra) : 0;
    for (int64_t c = warp0; c < nchunks; c += nwarps) {
        const int32_t k = chunk_row[c];
        const int64_t beg = chunk_beg[c];
        const int64_t end = min(rowptr[k + 1], beg + CHUNK);
        double acc[PL];
#pragma unroll
        for (int q = 0; q < PL; q++) acc[q] = 0.0;
        for (int64_t e0 = beg; e0 < end; e0 += 32) {
            const int64_t e = e0 + lane;
            const bool ok = e < end;
            int32_t myidx[MAXD - 1];
#pragma unroll
            for (int d = 0; d < MAXD - 1; d++)
                myidx[d] = (d < nother && ok) ? other[(int64_t)d * nnz + e] : 0;
            const double myv = ok ? val[e] : 0.0;
            const int cnt = (int)(end - e0 < 32 ? end - e0 : 32);
            for (int j = 0; j < cnt; j++) {
                const double v = __shfl_sync(0xffffffffu, myv, j);
                if (FAST3) {
                    const int ia = __shfl_sync(0xffffffffu, myidx[0], j);
                    const int ib = __shfl_sync(0xffffffffu, myidx[1], j);
                    const int Rb = f.R[1];
                    const double ua = f.U[0][(int64_t)ia * Ra + pa];
                    const double ubl = lane < Rb ? f.U[1][(int64_t)ib * Rb + lane] : 0.0;
                    const double w = v * ua;
#pragma unroll
                    for (int q = 0; q < PL; q++) {
                        const int pb = pb0 + q * pbstep;
                        const double ub = __shfl_sync(0xffffffffu, ubl, pb & 31);
                        acc[q] = fma(w, ub, acc[q]);
                    }
                } else {
                    int32_t ix[MAXD - 1];
#pragma unroll
                    for (int d = 0; d < MAXD - 1; d++)
                        ix[d] = __shfl_sync(0xffffffffu, myidx[d], j);
#pragma unroll
                    for (int q = 0; q < PL; q++) {
                        int p = lane + 32 * q;
                        if (p >= P) break;
                        double prod = v;
                        for (int d = 0; d < nother; d++) {
                            const int r = f.R[d];
                            const int pd = p % r;
                            p /= r;
                            prod *= f.U[d][(int64_t)ix[d] * r + pd];
                        }
                        acc[q] += prod;
                    }
                }
            }
        }
        const int32_t slot = chunk_slot[c];
        double *dst = slot < 0 ? Yc + (int64_t)k * P : Ypart + (int64_t)slot * P;
        if (FAST3) {
#pragma unroll
            for (int q = 0; q < PL; q++) {
                const int p = pa + Ra * (pb0 + q * pbstep);
                if (p < P) dst[p] = acc[q];
            }
        } else {
#pragma unroll
            for (int q = 0; q < PL; q++) {
                const int p = lane + 32 * q;
                if (p < P) dst[p] = acc[q];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// 3-way TTMc over the task list (even ranks RA, RB of the two other modes; P =
// RA * RB).  One warp per task.  Nonzeros go through in batches of 32:
//  * lane j loads nonzero j's two indices and value (coalesced); the batch
//    after next is already in registers, so these loads overlap compute;
//  * the two factor rows of every nonzero (RA + RB doubles) are copied into a
//    per-warp shared stage with 16-byte cp.async, double-buffered: batch b+1
//    is in flight while batch b is consumed;
//  * lane l owns BPL blocks of AW x BW Kronecker entries (p = pa + RA * pb);
//    per nonzero it reads AW + BW staged values and v, then AW*BW FMAs;
//  * a packed task walks whole rows: at each row boundary (from a register
//    window of 32 rowptr entries) the warp writes its row and restarts.
// Long rows arrive as pieces that write partial rows, summed in piece order by
// combine_partials_kernel: the output is deterministic, without atomics.
// ---------------------------------------------------------------------------
constexpr int T3_WARPS = 4;

__device__ __forceinline__ void sp_cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void sp_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void sp_cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int RA, int RB, int AW, int BW>
struct T3 {
    static constexpr int P = RA * RB;
    static constexpr int NBA = RA / AW, NBB = RB / BW, NBLK = NBA * NBB;
    static constexpr int BPL = (NBLK + 31) / 32;
    static constexpr int ROWW = RA + RB;  // staged doubles per nonzero
    static constexpr int PPN = ROWW / 2;  // 16-byte pieces per nonzero
    static constexpr int STAGE = 32 * ROWW;
    static constexpr int WARP_SMEM = 2 * STAGE + 32;  // doubles per warp
};

template <int RA, int RB, int AW, int BW>
__global__ void __launch_bounds__(T3_WARPS * 32) ttmc3_kernel(
    const int32_t *__restrict__ ia_arr, const int32_t *__restrict__ ib_arr,
    const double *__restrict__ val, const int64_t *__restrict__ rowptr, int64_t nrows,
    const int64_t *__restrict__ task_beg, const int64_t *__restrict__ task_end,
    const int32_t *__restrict__ task_row, const int32_t *__restrict__ task_slot, int64_t ntasks,
    const double *__restrict__ Ua, const double *__restrict__ Ub, double *__restrict__ Yc,
    double *__restrict__ Ypart) {
    using C = T3<RA, RB, AW, BW>;
    static_assert(RA % 2 == 0 && RB % 2 == 0 && RA % AW == 0 && RB % BW == 0, "tile shape");
    static_assert(AW == 1 || AW == 2, "AW");
    static_assert(BW == 2 || BW == 4, "BW");
    extern __shared__ __align__(16) double t3_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *stage0 = t3_smem + (size_t)wib * C::WARP_SMEM;
    double *vbuf = stage0 + 2 * C::STAGE;
    const int64_t gw = (int64_t)blockIdx.x * T3_WARPS + wib;
    const int64_t nw = (int64_t)gridDim.x * T3_WARPS;

    // Lane-owned blocks.
    int oa[C::BPL], ob[C::BPL];
    bool own[C::BPL];
#pragma unroll
    for (int q = 0; q < C::BPL; q++) {
        const int blk = lane + 32 * q;
        own[q] = blk < C::NBLK;
        oa[q] = own[q] ? AW * (blk % C::NBA) : 0;
        ob[q] = own[q] ? BW * (blk / C::NBA) : 0;
    }

    for (int64_t t = gw; t < ntasks; t += nw) {
        const int64_t beg = task_beg[t], end = task_end[t];
        int64_t row = task_row[t];
        const int32_t slot = task_slot[t];
        const int nb = (int)((end - beg + 31) / 32);

        // Row-boundary window: lane l holds rowptr[wbase + 1 + l].
        int64_t wbase = row;
        int64_t bnd_win = (wbase + 1 + lane <= nrows) ? rowptr[wbase + 1 + lane] : INT64_MAX;
        int wi = 0;

        auto load_idx = [&](int b, int &ia, int &ib, double &v) {
            const int64_t e = beg + 32 * (int64_t)b + lane;
            const bool ok = e < end;
            ia = ok ? ia_arr[e] : 0;
            ib = ok ? ib_arr[e] : 0;
            v = ok ? val[e] : 0.0;
        };
        auto issue = [&](int b, int ia, int ib) {
            double *st = stage0 + (b & 1) * C::STAGE;
            const int64_t e0 = beg + 32 * (int64_t)b;
            const int n_b = (int)(end - e0 < 32 ? end - e0 : 32);
#pragma unroll
            for (int s = 0; s < C::PPN; s++) {
                const int g = lane + 32 * s;
                const int jj = g / C::PPN, rem = g - jj * C::PPN;
                const int ija = __shfl_sync(0xffffffffu, ia, jj);
                const int ijb = __shfl_sync(0xffffffffu, ib, jj);
                if (jj < n_b) {
                    const double *src = rem < RA / 2 ? Ua + (int64_t)ija * RA + 2 * rem
                                                     : Ub + (int64_t)ijb * RB + 2 * (rem - RA / 2);
                    sp_cp_async16(st + jj * C::ROWW + 2 * rem, src);
                }
            }
            sp_cp_commit();
        };

        double acc[C::BPL][AW][BW];
#pragma unroll
        for (int q = 0; q < C::BPL; q++)
#pragma unroll
            for (int u = 0; u < AW; u++)
#pragma unroll
                for (int w = 0; w < BW; w++) acc[q][u][w] = 0.0;

        auto flush = [&](int64_t r) {
            double *dst = slot < 0 ? Yc + r * C::P : Ypart + (int64_t)slot * C::P;
#pragma unroll
            for (int q = 0; q < C::BPL; q++) {
                if (!own[q]) continue;
#pragma unroll
                for (int w = 0; w < BW; w++) {
                    double *d = dst + oa[q] + RA * (ob[q] + w);
                    if (AW == 2)
                        *reinterpret_cast<double2 *>(d) = make_double2(acc[q][0][w], acc[q][AW - 1][w]);
                    else
                        d[0] = acc[q][0][w];
#pragma unroll
                    for (int u = 0; u < AW; u++) acc[q][u][w] = 0.0;
                }
            }
        };

        int a_ia, a_ib;
        double a_v, cur_v, nxt_v = 0.0;
        load_idx(0, a_ia, a_ib, a_v);
        issue(0, a_ia, a_ib);
        cur_v = a_v;
        if (nb > 1) load_idx(1, a_ia, a_ib, a_v);
        int64_t next_bnd = __shfl_sync(0xffffffffu, bnd_win, 0);

        for (int b = 0; b < nb; b++) {
            if (b + 1 < nb) {
                issue(b + 1, a_ia, a_ib);
                nxt_v = a_v;
                if (b + 2 < nb) load_idx(b + 2, a_ia, a_ib, a_v);
                sp_cp_wait<1>();
            } else {
                sp_cp_wait<0>();
            }
            vbuf[lane] = cur_v;
            __syncwarp();
            const double *st = stage0 + (b & 1) * C::STAGE;
            const int64_t e0 = beg + 32 * (int64_t)b;
            const int n_b = (int)(end - e0 < 32 ? end - e0 : 32);
            for (int j = 0; j < n_b; j++) {
                if (e0 + j == next_bnd) {
                    flush(row);
                    row++;
                    if (++wi == 32) {
                        wbase += 32;
                        wi = 0;
                        bnd_win = (wbase + 1 + lane <= nrows) ? rowptr[wbase + 1 + lane] : INT64_MAX;
                    }
                    next_bnd = __shfl_sync(0xffffffffu, bnd_win, wi);
                }
                const double v = vbuf[j];
                const double *srow = st + j * C::ROWW;
#pragma unroll
                for (int q = 0; q < C::BPL; q++) {
                    if (!own[q]) continue;
                    double wa[AW], ub[BW];
                    if (AW == 2) {
                        const double2 x = *reinterpret_cast<const double2 *>(srow + oa[q]);
                        wa[0] = v * x.x;
                        wa[AW - 1] = v * x.y;
                    } else {
                        wa[0] = v * srow[oa[q]];
                    }
#pragma unroll
                    for (int w = 0; w < BW; w += 2) {
                        const double2 y = *reinterpret_cast<const double2 *>(srow + RA + ob[q] + w);
                        ub[w] = y.x;
                        ub[w + 1] = y.y;
                    }
#pragma unroll
                    for (int u = 0; u < AW; u++)
#pragma unroll
                        for (int w = 0; w < BW; w++) acc[q][u][w] = fma(wa[u], ub[w], acc[q][u][w]);
                }
            }
            cur_v = nxt_v;
            __syncwarp();
        }
        flush(row);
    }
}

// Yc[row] = sum of its partial rows, in chunk order (deterministic).
__global__ void combine_partials_kernel(const double *__restrict__ Ypart,
                                        const int32_t *__restrict__ multi_row,
                                        const int32_t *__restrict__ multi_first,
                                        const int32_t *__restrict__ multi_count, int64_t nmulti,
                                        int P, double *__restrict__ Yc) {
    for (int64_t m = blockIdx.x; m < nmulti; m += gridDim.x) {
        const int32_t k = multi_row[m];
        const int64_t first = multi_first[m];
        const int cnt = multi_count[m];
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            double s = 0.0;
            for (int c = 0; c < cnt; c++) s += Ypart[(first + c) * P + p];
            Yc[(int64_t)k * P + p] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// ttmc_mTL / ttmc_mTR on the FP64 tensor-core path (mma.sync m8n8k4 .f64).
// Operand fragments: A[g][t] and B[t][g] with g = lane / 4, t = lane % 4;
// the 8 x 8 result D[g][2t + {0, 1}].  Staged shared operands use a pitch of
// 4 (mod 16) doubles so a half-warp's fragment loads hit distinct banks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sp_dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// out[rows[k] * Rn + r] = sum_p Yc[k, p] L[p + P r].  One warp per 8 compact
// rows; NTL = ceil(Rn / 8) output tiles.  L staged in shared memory (pitch
// 8 NTL + 4) when LSM, else read through the read-only cache.
template <int NTL, bool LSM>
__global__ void __launch_bounds__(256) mtl_mma_kernel(const double *__restrict__ Yc,
                                                      const int32_t *__restrict__ rows,
                                                      int64_t nrows, int P,
                                                      const double *__restrict__ L, int Rn,
                                                      double *__restrict__ out) {
    constexpr int LDL = 8 * NTL + 4;
    extern __shared__ __align__(16) double Ls[];
    const int P4 = (P + 3) & ~3;
    if (LSM) {
        for (int e = threadIdx.x; e < P4 * LDL; e += blockDim.x) {
            const int p = e / LDL, r = e - p * LDL;
            Ls[e] = (p < P && r < Rn) ? L[p + (int64_t)P * r] : 0.0;
        }
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t mtiles = (nrows + 7) / 8;
    const int ksteps = P4 / 4;
    for (int64_t mt = warp0; mt < mtiles; mt += nwarps) {
        const int64_t k = 8 * mt + g;
        const bool okr = k < nrows;
        const double *y = Yc + (okr ? k : 0) * (int64_t)P;
        double acc[NTL][2];
#pragma unroll
        for (int j = 0; j < NTL; j++) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll 8
        for (int kk = 0; kk < ksteps; kk++) {
            const int p = 4 * kk + t;
            const double a = (okr && p < P) ? y[p] : 0.0;
#pragma unroll
            for (int j = 0; j < NTL; j++) {
                const int r = 8 * j + g;
                const double b = LSM ? Ls[p * LDL + r]
                                     : ((p < P && r < Rn) ? __ldg(L + p + (int64_t)P * r) : 0.0);
                sp_dmma(acc[j][0], acc[j][1], a, b);
            }
        }
        if (okr) {
            double *o = out + (int64_t)rows[k] * Rn;
#pragma unroll
            for (int j = 0; j < NTL; j++) {
                const int r = 8 * j + 2 * t;
                if (r < Rn) o[r] = acc[j][0];
                if (r + 1 < Rn) o[r + 1] = acc[j][1];
            }
        }
    }
}

// mTR partials: part[blk][p + P r] = sum over the block's compact rows k of
// Yc[k, p] U(rows[k], r) (U transposed: row i at U + i Rn).  The block's rows
// go through in batches of 64 whose U rows are staged in shared memory; warp
// w owns p-tiles w, w + 8, ... (up to 4 at a time).
template <int NTL>
__global__ void __launch_bounds__(256) mtr_mma_kernel(const double *__restrict__ Yc,
                                                      const int32_t *__restrict__ rows,
                                                      int64_t nrows, int P,
                                                      const double *__restrict__ U, int Rn,
                                                      int64_t rows_per_block,
                                                      double *__restrict__ part) {
    constexpr int LDU = 8 * NTL + 4, KB = 64, MG = 4;
    __shared__ __align__(16) double Us[KB * LDU];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int64_t k0 = blockIdx.x * rows_per_block;
    const int64_t k1 = min(nrows, k0 + rows_per_block);
    const int ptiles = (P + 7) / 8;
    double *pb = part + (int64_t)blockIdx.x * P * Rn;
    for (int mbase = 0; mbase < ptiles; mbase += 8 * MG) {
        double acc[MG][NTL][2];
#pragma unroll
        for (int m = 0; m < MG; m++)
#pragma unroll
            for (int j = 0; j < NTL; j++) acc[m][j][0] = acc[m][j][1] = 0.0;
        for (int64_t kb = k0; kb < k1; kb += KB) {
            __syncthreads();
            for (int e = threadIdx.x; e < KB * LDU; e += blockDim.x) {
                const int b = e / LDU, c = e - b * LDU;
                const int64_t k = kb + b;
                Us[e] = (k < k1 && c < Rn) ? U[(int64_t)rows[k] * Rn + c] : 0.0;
            }
            __syncthreads();
            const int kn = (int)min((int64_t)KB, k1 - kb);
            const int ks_end = (kn + 3) / 4;
            for (int ks = 0; ks < ks_end; ks++) {
                const int bl = 4 * ks + t;
                const int64_t k = kb + bl;
                const bool okk = bl < kn;
                double bv[NTL];
#pragma unroll
                for (int j = 0; j < NTL; j++) bv[j] = Us[bl * LDU + 8 * j + g];
#pragma unroll
                for (int m = 0; m < MG; m++) {
                    const int mt = mbase + w + 8 * m;
                    const int p = 8 * mt + g;
                    const double a = (okk && mt < ptiles && p < P) ? Yc[k * P + p] : 0.0;
#pragma unroll
                    for (int j = 0; j < NTL; j++) sp_dmma(acc[m][j][0], acc[m][j][1], a, bv[j]);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < MG; m++) {
            const int mt = mbase + w + 8 * m;
            const int p = 8 * mt + g;
            if (mt >= ptiles || p >= P) continue;
#pragma unroll
            for (int j = 0; j < NTL; j++) {
                const int r = 8 * j + 2 * t;
                if (r < Rn) pb[p + (int64_t)P * r] = acc[m][j][0];
                if (r + 1 < Rn) pb[p + (int64_t)P * (r + 1)] = acc[m][j][1];
            }
        }
    }
}

// Y[rows[k], :] = Yc[k, :] for the full (I_n x P) output.
__global__ void scatter_rows_kernel(const double *__restrict__ Yc,
                                    const int32_t *__restrict__ rows, int64_t nrows, int P,
                                    double *__restrict__ Y) {
    const int64_t n = nrows * P;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / P, p = e - k * P;
        Y[(int64_t)rows[k] * P + p] = Yc[e];
    }
}

__global__ void sum_blocks_kernel(const double *__restrict__ part, int nblk, int64_t n,
                                  double *__restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(int64_t)b * n + e];
        out[e] = s;
    }
}

int64_t kron_len(const int64_t *R, int ndim, int mode) {
    int64_t P = 1;
    for (int m = 0; m < ndim; m++)
        if (m != mode) P *= R[m];
    return P;
}

void build_mode(dt_ctx *ctx, dt_sptensor *sp, int n, const std::vector<DevMem> &idx32,
                const double *vals_dev) {
    ModeCopy &mc = sp->modes[n];
    const int64_t nnz = sp->nnz;
    const int nd = sp->ndim;
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceil_div(nnz, 256), 8 * ctx->num_sms));
    // Stable radix sort of (row index, nonzero id).
    DevMem ids(ctx, nnz * sizeof(int32_t)), keys_out(ctx, nnz * sizeof(int32_t)),
        perm(ctx, nnz * sizeof(int32_t));
    DT_LAUNCH(ctx, iota_kernel, blocks, 256, 0, ids.as<int32_t>(), nnz);
    int bits = 1;
    while ((int64_t(1) << bits) < sp->shape[n]) bits++;
    size_t tmp_bytes = 0;
    DT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, idx32[n].as<int32_t>(),
                                            keys_out.as<int32_t>(), ids.as<int32_t>(),
                                            perm.as<int32_t>(), (int)nnz, 0, bits, ctx->stream));
    DevMem tmp(ctx, tmp_bytes);
    DT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, idx32[n].as<int32_t>(),
                                            keys_out.as<int32_t>(), ids.as<int32_t>(),
                                            perm.as<int32_t>(), (int)nnz, 0, bits, ctx->stream));
    ctx->launches += 1;
    mc.other.alloc(ctx, (size_t)(nd - 1) * nnz * sizeof(int32_t));
    int d = 0;
    for (int m = 0; m < nd; m++) {
        if (m == n) continue;
        DT_LAUNCH(ctx, gather_kernel<int32_t>, blocks, 256, 0, idx32[m].as<int32_t>(),
                  perm.as<int32_t>(), nnz, mc.other.as<int32_t>() + (int64_t)d * nnz);
        d++;
    }
    mc.val.alloc(ctx, nnz * sizeof(double));
    DT_LAUNCH(ctx, gather_kernel<double>, blocks, 256, 0, vals_dev, perm.as<int32_t>(), nnz,
              mc.val.as<double>());
    // Row structure and chunk lists on the host (construction-time only).
    std::vector<int32_t> hk((size_t)nnz);
    DT_CUDA(cudaMemcpyAsync(hk.data(), keys_out.get(), nnz * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> rows;
    std::vector<int64_t> rowptr;
    for (int64_t e = 0; e < nnz; e++) {
        if (e == 0 || hk[e] != hk[e - 1]) {
            rows.push_back(hk[e]);
            rowptr.push_back(e);
        }
    }
    rowptr.push_back(nnz);
    mc.nrows = (int64_t)rows.size();
    std::vector<int32_t> crow, cslot, mrow, mfirst, mcount;
    std::vector<int64_t> cbeg;
    int64_t slots = 0;
    for (int64_t k = 0; k < mc.nrows; k++) {
        const int64_t c = rowptr[k + 1] - rowptr[k];
        const int64_t nch = (c + CHUNK - 1) / CHUNK;
        if (nch > 1) {
            mrow.push_back((int32_t)k);
            mfirst.push_back((int32_t)slots);
            mcount.push_back((int32_t)nch);
        }
        for (int64_t j = 0; j < nch; j++) {
            crow.push_back((int32_t)k);
            cbeg.push_back(rowptr[k] + j * CHUNK);
            cslot.push_back(nch > 1 ? (int32_t)(slots + j) : -1);
        }
        if (nch > 1) slots += nch;
    }
    mc.nchunks = (int64_t)crow.size();
    mc.nslots = slots;
    mc.nmulti = (int64_t)mrow.size();
    // Tasks of the 3-way kernel.
    struct Task {
        int64_t beg, end;
        int32_t row, slot;
    };
    std::vector<Task> tasks;
    std::vector<int32_t> tmrow, tmfirst, tmcount;
    int64_t tslots = 0;
    {
        int64_t pack_beg = -1;
        int32_t pack_row = 0;
        auto close_pack = [&](int64_t e) {
            if (pack_beg >= 0) tasks.push_back({pack_beg, e, pack_row, -1});
            pack_beg = -1;
        };
        for (int64_t k = 0; k < mc.nrows; k++) {
            const int64_t b = rowptr[k], c = rowptr[k + 1] - b;
            if (c > TASK_PACK) {
                close_pack(b);
                const int64_t np = (c + TASK_PIECE - 1) / TASK_PIECE;
                if (np > 1) {
                    tmrow.push_back((int32_t)k);
                    tmfirst.push_back((int32_t)tslots);
                    tmcount.push_back((int32_t)np);
                }
                for (int64_t j = 0; j < np; j++)
                    tasks.push_back({b + j * TASK_PIECE, std::min(b + c, b + (j + 1) * TASK_PIECE),
                                     (int32_t)k, np > 1 ? (int32_t)(tslots + j) : -1});
                if (np > 1) tslots += np;
                continue;
            }
            if (pack_beg >= 0 && b + c - pack_beg > TASK_PACK) close_pack(b);
            if (pack_beg < 0) {
                pack_beg = b;
                pack_row = (int32_t)k;
            }
        }
        close_pack(nnz);
        std::stable_sort(tasks.begin(), tasks.end(), [](const Task &a, const Task &b) {
            return a.end - a.beg > b.end - b.beg;
        });
    }
    mc.ntasks = (int64_t)tasks.size();
    mc.tslots = tslots;
    mc.tmulti = (int64_t)tmrow.size();
    std::vector<int64_t> tbeg(tasks.size()), tend(tasks.size());
    std::vector<int32_t> trow(tasks.size()), tslot(tasks.size());
    for (size_t i = 0; i < tasks.size(); i++) {
        tbeg[i] = tasks[i].beg;
        tend[i] = tasks[i].end;
        trow[i] = tasks[i].row;
        tslot[i] = tasks[i].slot;
    }
    auto up = [&](DevMem &dst, const void *src, size_t bytes) {
        dst.alloc(ctx, std::max<size_t>(bytes, 8));
        if (bytes)
            DT_CUDA(cudaMemcpyAsync(dst.get(), src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    };
    up(mc.rows, rows.data(), rows.size() * sizeof(int32_t));
    up(mc.rowptr, rowptr.data(), rowptr.size() * sizeof(int64_t));
    up(mc.chunk_row, crow.data(), crow.size() * sizeof(int32_t));
    up(mc.chunk_beg, cbeg.data(), cbeg.size() * sizeof(int64_t));
    up(mc.chunk_slot, cslot.data(), cslot.size() * sizeof(int32_t));
    up(mc.multi_row, mrow.data(), mrow.size() * sizeof(int32_t));
    up(mc.multi_first, mfirst.data(), mfirst.size() * sizeof(int32_t));
    up(mc.multi_count, mcount.data(), mcount.size() * sizeof(int32_t));
    up(mc.task_beg, tbeg.data(), tbeg.size() * sizeof(int64_t));
    up(mc.task_end, tend.data(), tend.size() * sizeof(int64_t));
    up(mc.task_row, trow.data(), trow.size() * sizeof(int32_t));
    up(mc.task_slot, tslot.data(), tslot.size() * sizeof(int32_t));
    up(mc.tmulti_row, tmrow.data(), tmrow.size() * sizeof(int32_t));
    up(mc.tmulti_first, tmfirst.data(), tmfirst.size() * sizeof(int32_t));
    up(mc.tmulti_count, tmcount.data(), tmcount.size() * sizeof(int32_t));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
}

template <int PL, bool FAST3>
void launch_rows(dt_ctx *ctx, const ModeCopy &mc, int nother, int64_t nnz, const FactorSet &f,
                 int P, double *Yc, double *Ypart) {
    const int64_t warps = mc.nchunks;
    const unsigned blocks =
        std::max(1u, std::min<unsigned>(ceil_div(warps, 8), 32u * (unsigned)ctx->num_sms));
    DT_LAUNCH(ctx, (ttmc_rows_kernel<PL, FAST3>), blocks, 256, 0, mc.other.as<int32_t>(),
              mc.val.as<double>(), nnz, nother, mc.rowptr.as<int64_t>(),
              mc.chunk_row.as<int32_t>(), mc.chunk_beg.as<int64_t>(),
              mc.chunk_slot.as<int32_t>(), mc.nchunks, f, P, Yc, Ypart);
}

template <int RA, int RB, int AW, int BW>
void launch_t3(dt_ctx *ctx, const ModeCopy &mc, int64_t nnz, const FactorSet &f, double *Yc,
               double *Ypart) {
    using C = T3<RA, RB, AW, BW>;
    const size_t smem = (size_t)T3_WARPS * C::WARP_SMEM * sizeof(double);
    auto kern = ttmc3_kernel<RA, RB, AW, BW>;
    smem_limit(ctx, kern, smem);
    const int per_sm = std::max<int>(1, std::min<int>(8, (int)((220 * 1024) / smem)));
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((mc.ntasks + T3_WARPS - 1) / T3_WARPS, (int64_t)per_sm * ctx->num_sms));
    DT_LAUNCH(ctx, kern, blocks, T3_WARPS * 32, smem, mc.other.as<int32_t>(),
              mc.other.as<int32_t>() + nnz, mc.val.as<double>(), mc.rowptr.as<int64_t>(),
              mc.nrows, mc.task_beg.as<int64_t>(), mc.task_end.as<int64_t>(),
              mc.task_row.as<int32_t>(), mc.task_slot.as<int32_t>(), mc.ntasks, f.U[0], f.U[1],
              Yc, Ypart);
}

// The 3-way task kernel for the rank pairs it is instantiated for; false if
// (Ra, Rb) is not one of them.
bool ttmc3_dispatch(dt_ctx *ctx, const ModeCopy &mc, int64_t nnz, const FactorSet &f, double *Yc,
                    double *Ypart) {
    const int a = f.R[0], b = f.R[1];
#define DT_T3(RA, RB, AW, BW)                                        \
    if (a == RA && b == RB) {                                        \
        launch_t3<RA, RB, AW, BW>(ctx, mc, nnz, f, Yc, Ypart);       \
        return true;                                                 \
    }
    DT_T3(16, 16, 2, 4)
    DT_T3(8, 8, 1, 2)
    DT_T3(32, 32, 2, 4)
    DT_T3(16, 8, 1, 4)
    DT_T3(8, 16, 1, 4)
    DT_T3(10, 10, 1, 2)
    DT_T3(12, 12, 1, 4)
    DT_T3(4, 4, 1, 2)
#undef DT_T3
    return false;
}

}  // namespace

// Compact Y_(n): Yc is nrows x P row-major (row k = mode-n row mc.rows[k]).
void sp_ttmc_compact(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut_dev,
                     const int64_t *R, int mode, double *Yc, LaunchTimer *timer = nullptr) {
    const ModeCopy &mc = sp->modes[mode];
    const int nd = sp->ndim;
    const int64_t P64 = kron_len(R, nd, mode);
    DT_CHECK_ARG(P64 <= 1024, "sparse TTMc: prod of the other ranks (%lld) exceeds 1024",
                 (long long)P64);
    const int P = (int)P64;
    FactorSet f{};
    int d = 0;
    for (int m = 0; m < nd; m++) {
        if (m == mode) continue;
        f.U[d] = Ut_dev[m];
        f.R[d] = (int)R[m];
        d++;
    }
    if (nd == 3 && mc.ntasks > 0) {
        DevMem tpart(ctx, std::max<int64_t>(mc.tslots, 1) * P * sizeof(double));
        if (timer) timer->begin();
        if (ttmc3_dispatch(ctx, mc, sp->nnz, f, Yc, tpart.as<double>())) {
            if (mc.tmulti > 0) {
                const unsigned blocks = (unsigned)std::min<int64_t>(mc.tmulti, 65535);
                DT_LAUNCH(ctx, combine_partials_kernel, blocks, 256, 0, tpart.as<double>(),
                          mc.tmulti_row.as<int32_t>(), mc.tmulti_first.as<int32_t>(),
                          mc.tmulti_count.as<int32_t>(), mc.tmulti, P, Yc);
            }
            if (timer) {
                double bytes = (double)sp->nnz * (4.0 * (nd - 1) + 8.0) + (double)mc.nrows * P * 8.0;
                for (int m = 0; m < nd; m++)
                    if (m != mode) bytes += (double)sp->shape[m] * R[m] * 8.0;
                timer->end(bytes);
            }
            return;
        }
    }
    DevMem part(ctx, std::max<int64_t>(mc.nslots, 1) * P * sizeof(double));
    if (timer) timer->begin();
    const bool fast3 = nd == 3 && f.R[0] <= 32 && (32 % f.R[0]) == 0 && f.R[1] <= 32;
    const int PL = (P + 31) / 32;
    if (fast3) {
        if (PL <= 1) launch_rows<1, true>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 2) launch_rows<2, true>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 4) launch_rows<4, true>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 8) launch_rows<8, true>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 16) launch_rows<16, true>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else launch_rows<32, true>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    } else {
        if (PL <= 1) launch_rows<1, false>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 2) launch_rows<2, false>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 4) launch_rows<4, false>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 8) launch_rows<8, false>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else if (PL <= 16) launch_rows<16, false>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
        else launch_rows<32, false>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    }
    if (mc.nmulti > 0) {
        const unsigned blocks = (unsigned)std::min<int64_t>(mc.nmulti, 65535);
        DT_LAUNCH(ctx, combine_partials_kernel, blocks, 256, 0, part.as<double>(),
                  mc.multi_row.as<int32_t>(), mc.multi_first.as<int32_t>(),
                  mc.multi_count.as<int32_t>(), mc.nmulti, P, Yc);
    }
    if (timer) {
        // Algorithmic bytes of the TTMc: the mode-sorted nonzeros (int32 indices
        // of the other modes + FP64 value), each other factor read once, and
        // the compact Y_(n) rows written.
        double bytes = (double)sp->nnz * (4.0 * (nd - 1) + 8.0) + (double)mc.nrows * P * 8.0;
        for (int m = 0; m < nd; m++)
            if (m != mode) bytes += (double)sp->shape[m] * R[m] * 8.0;
        timer->end(bytes);
    }
}

void sp_mtr(dt_ctx *ctx, const dt_sptensor *sp, const double *Yc, int mode, int P,
            const double *Un, int Rn, double *L) {
    const ModeCopy &mc = sp->modes[mode];
    DT_CHECK_ARG(Rn <= 32, "sparse ttmc_mTR: R_n (%d) must be <= 32", Rn);
    const int64_t target = 2LL * ctx->num_sms;
    const int64_t rpb = std::max<int64_t>(64, (mc.nrows + target - 1) / target);
    const int nblk = (int)std::max<int64_t>(1, (mc.nrows + rpb - 1) / rpb);
    DevMem part(ctx, (size_t)nblk * P * Rn * sizeof(double));
    const int ntl = (Rn + 7) / 8;
#define DT_MTR(N)                                                                          \
    DT_LAUNCH(ctx, mtr_mma_kernel<N>, nblk, 256, 0, Yc, mc.rows.as<int32_t>(), mc.nrows, P, \
              Un, Rn, rpb, part.as<double>())
    if (ntl == 1) DT_MTR(1);
    else if (ntl == 2) DT_MTR(2);
    else if (ntl == 3) DT_MTR(3);
    else DT_MTR(4);
#undef DT_MTR
    const int64_t n = (int64_t)P * Rn;
    DT_LAUNCH(ctx, sum_blocks_kernel, std::max(1u, ceil_div(n, 256)), 256, 0,
              part.as<double>(), nblk, n, L);
}

void sp_mtl(dt_ctx *ctx, const dt_sptensor *sp, const double *Yc, int mode, int P,
            const double *L, int Rn, double *out) {
    const ModeCopy &mc = sp->modes[mode];
    DT_CHECK_ARG(Rn <= 32, "sparse ttmc_mTL: R_n (%d) must be <= 32", Rn);
    DT_CUDA(cudaMemsetAsync(out, 0, sp->shape[mode] * Rn * sizeof(double), ctx->stream));
    const int ntl = (Rn + 7) / 8;
    const size_t smem = (size_t)((P + 3) & ~3) * (8 * ntl + 4) * sizeof(double);
    const bool lsm = smem <= 160 * 1024;
    const unsigned blocks = std::max(
        1u, std::min<unsigned>(ceil_div((mc.nrows + 7) / 8, 8), 4u * (unsigned)ctx->num_sms));
#define DT_MTL(N, S)                                                                         \
    do {                                                                                     \
        auto kern = mtl_mma_kernel<N, S>;                                                    \
        const size_t sm = S ? smem : 0;                                                      \
        smem_limit(ctx, kern, sm);                                                           \
        DT_LAUNCH(ctx, kern, blocks, 256, sm, Yc, mc.rows.as<int32_t>(), mc.nrows, P, L, Rn, \
                  out);                                                                      \
    } while (0)
    if (lsm) {
        if (ntl == 1) DT_MTL(1, true);
        else if (ntl == 2) DT_MTL(2, true);
        else if (ntl == 3) DT_MTL(3, true);
        else DT_MTL(4, true);
    } else {
        if (ntl == 1) DT_MTL(1, false);
        else if (ntl == 2) DT_MTL(2, false);
        else if (ntl == 3) DT_MTL(3, false);
        else DT_MTL(4, false);
    }
#undef DT_MTL
}

void detach_sptensors(dt_ctx *ctx) {
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (dt_sptensor *sp : ctx->sptensors) {
        sp->modes.clear();
        sp->ctx = nullptr;
    }
    ctx->sptensors.clear();
}

}  // namespace dt

using namespace dt;

namespace {

struct FactorUpload {
    std::vector<DevView> views;
    const double *ptrs[dt::MAXD];
};

void upload_factors(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                    const int64_t *R, FactorUpload &fu) {
    DT_CHECK_ARG(Ut && R, "sparse: null factors");
    fu.views.reserve(sp->ndim);
    for (int m = 0; m < sp->ndim; m++) {
        DT_CHECK_ARG(R[m] >= 1 && R[m] <= sp->shape[m], "sparse: bad rank R[%d] = %lld", m,
                     (long long)R[m]);
        fu.views.emplace_back(ctx, Ut[m], sp->shape[m] * R[m] * sizeof(double), true, false);
        fu.ptrs[m] = fu.views.back().as<double>();
    }
}

void check_sp(const dt_ctx *ctx, const dt_sptensor *sp, int mode) {
    check_ctx(ctx);
    DT_CHECK_ARG(sp, "null dt_sptensor");
    DT_CHECK_ARG(sp->ctx == ctx, sp->ctx ? "dt_sptensor belongs to another dt_ctx"
                                         : "dt_sptensor's dt_ctx was destroyed");
    DT_CHECK_ARG(mode >= 0 && mode < sp->ndim, "sparse: mode %d out of range", mode);
}

}  // namespace

extern "C" {

int dt_sptensor_create(dt_ctx *ctx, int64_t nnz, int ndim, const int64_t *const *idx,
                       const double *vals, const int64_t *shape, dt_sptensor **out) {
    return guard([&] {
        check_ctx(ctx);
        DT_CHECK_ARG(out && shape, "dt_sptensor_create: null argument");
        DT_CHECK_ARG(ndim >= 2 && ndim <= MAXD, "dt_sptensor_create: ndim %d not in [2, %d]",
                     ndim, MAXD);
        DT_CHECK_ARG(nnz >= 1 && nnz < (int64_t(1) << 31),
                     "dt_sptensor_create: nnz %lld not in [1, 2^31)", (long long)nnz);
        DT_CHECK_ARG(idx && vals, "dt_sptensor_create: null indices or values");
        for (int m = 0; m < ndim; m++)
            DT_CHECK_ARG(shape[m] >= 1 && shape[m] < (int64_t(1) << 31) && idx[m],
                         "dt_sptensor_create: bad mode %d", m);
        DT_CUDA(cudaSetDevice(ctx->device));
        auto *sp = new dt_sptensor();
        try {
            sp->ctx = ctx;
            sp->ndim = ndim;
            sp->nnz = nnz;
            for (int m = 0; m < ndim; m++) sp->shape[m] = shape[m];
            DevMem bad(ctx, sizeof(int));
            DT_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), ctx->stream));
            std::vector<DevMem> idx32(ndim);
            const unsigned blocks =
                std::max(1u, std::min<unsigned>(ceil_div(nnz, 256), 8 * ctx->num_sms));
            for (int m = 0; m < ndim; m++) {
                DevView src(ctx, idx[m], nnz * sizeof(int64_t), true, false);
                idx32[m].alloc(ctx, nnz * sizeof(int32_t));
                DT_LAUNCH(ctx, narrow_index_kernel, blocks, 256, 0, src.as<int64_t>(), nnz,
                          shape[m], idx32[m].as<int32_t>(), bad.as<int>());
                DT_CUDA(cudaStreamSynchronize(ctx->stream));
            }
            int hbad = 0;
            DT_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            DT_CUDA(cudaStreamSynchronize(ctx->stream));
            if (hbad) fail(DT_ERR_ARG, "dt_sptensor_create: an index is outside the shape");
            DevView v(ctx, vals, nnz * sizeof(double), true, false);
            DevMem s(ctx, sizeof(double));
            sumsq(ctx, v.ptr(), DT_F64, nnz, s.as<double>());
            double h = 0.0;
            DT_CUDA(cudaMemcpyAsync(&h, s.get(), sizeof(double), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            sp->modes.resize(ndim);
            for (int m = 0; m < ndim; m++) build_mode(ctx, sp, m, idx32, v.as<double>());
            DT_CUDA(cudaStreamSynchronize(ctx->stream));
            sp->fnorm = std::sqrt(h);
        } catch (...) {
            delete sp;
            throw;
        }
        ctx->sptensors.insert(sp);
        *out = sp;
    });
}

int dt_sptensor_destroy(dt_sptensor *sp) {
    return guard([&] {
        if (!sp) return;
        if (sp->ctx) {
            cudaSetDevice(sp->ctx->device);
            cudaStreamSynchronize(sp->ctx->stream);
            sp->ctx->sptensors.erase(sp);
        }
        delete sp;
    });
}

int dt_sp_fnorm(dt_ctx *ctx, const dt_sptensor *sp, double *out) {
    return guard([&] {
        check_sp(ctx, sp, 0);
        DT_CHECK_ARG(out, "dt_sp_fnorm: null output");
        *out = sp->fnorm;
    });
}

int dt_sp_ttmc_rows(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                    const int64_t *R, int mode, double *Y) {
    return guard([&] {
        check_sp(ctx, sp, mode);
        DT_CUDA(cudaSetDevice(ctx->device));
        FactorUpload fu;
        upload_factors(ctx, sp, Ut, R, fu);
        const ModeCopy &mc = sp->modes[mode];
        const int64_t P = kron_len(R, sp->ndim, mode);
        DevMem Yc(ctx, std::max<int64_t>(mc.nrows, 1) * P * sizeof(double));
        sp_ttmc_compact(ctx, sp, fu.ptrs, R, mode, Yc.as<double>());
        // Scatter compact rows into the full I_n x P row-major output.
        DevView y(ctx, Y, sp->shape[mode] * P * sizeof(double), false, true);
        DT_CUDA(cudaMemsetAsync(y.ptr(), 0, sp->shape[mode] * P * sizeof(double), ctx->stream));
        const unsigned blocks = std::max(
            1u, std::min<unsigned>(ceil_div(mc.nrows * P, 256), 8u * (unsigned)ctx->num_sms));
        DT_LAUNCH(ctx, scatter_rows_kernel, blocks, 256, 0, Yc.as<double>(),
                  mc.rows.as<int32_t>(), mc.nrows, (int)P, y.as<double>());
        y.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_sp_ttmc_mTR(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                   const int64_t *R, int mode, double *L) {
    return guard([&] {
        check_sp(ctx, sp, mode);
        DT_CUDA(cudaSetDevice(ctx->device));
        FactorUpload fu;
        upload_factors(ctx, sp, Ut, R, fu);
        const ModeCopy &mc = sp->modes[mode];
        const int P = (int)kron_len(R, sp->ndim, mode);
        DevMem Yc(ctx, std::max<int64_t>(mc.nrows, 1) * P * sizeof(double));
        sp_ttmc_compact(ctx, sp, fu.ptrs, R, mode, Yc.as<double>());
        DevView l(ctx, L, (size_t)P * R[mode] * sizeof(double), false, true);
        sp_mtr(ctx, sp, Yc.as<double>(), mode, P, fu.ptrs[mode], (int)R[mode], l.as<double>());
        l.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_sp_ttmc_mTL(dt_ctx *ctx, const dt_sptensor *sp, const double *const *Ut,
                   const int64_t *R, int mode, const double *L, double *out) {
    return guard([&] {
        check_sp(ctx, sp, mode);
        DT_CUDA(cudaSetDevice(ctx->device));
        FactorUpload fu;
        upload_factors(ctx, sp, Ut, R, fu);
        const ModeCopy &mc = sp->modes[mode];
        const int P = (int)kron_len(R, sp->ndim, mode);
        DevMem Yc(ctx, std::max<int64_t>(mc.nrows, 1) * P * sizeof(double));
        sp_ttmc_compact(ctx, sp, fu.ptrs, R, mode, Yc.as<double>());
        DevView l(ctx, L, (size_t)P * R[mode] * sizeof(double), true, false);
        DevView o(ctx, out, sp->shape[mode] * R[mode] * sizeof(double), false, true);
        sp_mtl(ctx, sp, Yc.as<double>(), mode, P, l.as<double>(), (int)R[mode], o.as<double>());
        o.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_sp_hooi(dt_ctx *ctx, const dt_sptensor *sp, const int64_t *R, int max_sweeps,
               double *const *Ut, double *G, dt_hooi_report *report) {
    return guard([&] {
        check_sp(ctx, sp, 0);
        DT_CHECK_ARG(max_sweeps >= 0, "dt_sp_hooi: max_sweeps must be >= 0");
        DT_CUDA(cudaSetDevice(ctx->device));
        if (report) std::memset(report, 0, sizeof(*report));
        const int nd = sp->ndim;
        const int64_t launches0 = ctx->launches;
        std::vector<DevView> views;
        views.reserve(nd);
        const double *ptrs[MAXD];
        for (int m = 0; m < nd; m++) {
            DT_CHECK_ARG(Ut && Ut[m] && R[m] >= 1 && R[m] <= sp->shape[m] && R[m] <= 32,
                         "dt_sp_hooi: bad factor / rank for mode %d", m);
            views.emplace_back(ctx, Ut[m], sp->shape[m] * R[m] * sizeof(double), true, true);
            ptrs[m] = views.back().as<double>();
        }
        int64_t maxYc = 1;
        for (int m = 0; m < nd; m++)
            maxYc = std::max<int64_t>(maxYc, sp->modes[m].nrows * kron_len(R, nd, m));
        DevMem Yc(ctx, maxYc * sizeof(double));
        DevMem L(ctx, 1024 * 32 * sizeof(double));
        LaunchTimer timer(ctx, true);  // TTMc launches, reported as ttm_x_*
        DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
        for (int it = 0; it < max_sweeps; it++) {
            for (int n = 0; n < nd; n++) {
                const int P = (int)kron_len(R, nd, n);
                sp_ttmc_compact(ctx, sp, ptrs, R, n, Yc.as<double>(), &timer);
                sp_mtr(ctx, sp, Yc.as<double>(), n, P, ptrs[n], (int)R[n], L.as<double>());
                sp_mtl(ctx, sp, Yc.as<double>(), n, P, L.as<double>(), (int)R[n],
                       const_cast<double *>(ptrs[n]));
                orth2_rows(ctx, const_cast<double *>(ptrs[n]), R[n], sp->shape[n]);
            }
        }
        const int last = nd - 1;
        const int P = (int)kron_len(R, nd, last);
        sp_ttmc_compact(ctx, sp, ptrs, R, last, Yc.as<double>());
        sp_mtr(ctx, sp, Yc.as<double>(), last, P, ptrs[last], (int)R[last], L.as<double>());
        DevMem g2(ctx, sizeof(double));
        sumsq(ctx, L.get(), DT_F64, (int64_t)P * R[last], g2.as<double>());
        DT_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
        double hg2 = 0.0;
        DT_CUDA(cudaMemcpyAsync(&hg2, g2.get(), sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
        if (G) {
            DevView g(ctx, G, (size_t)P * R[last] * sizeof(double), false, true);
            DT_CUDA(cudaMemcpyAsync(g.ptr(), L.get(), (size_t)P * R[last] * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
            g.finish();
        }
        for (auto &v : views) v.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        float ms = 0.f;
        DT_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        if (report) {
            report->sweeps = max_sweeps;
            report->x_norm = sp->fnorm;
            report->g_norm = std::sqrt(hg2);
            report->residual =
                std::sqrt(std::max(0.0, 1.0 - hg2 / (sp->fnorm * sp->fnorm)));
            report->device_ms = ms;
            report->kernel_launches = (int)(ctx->launches - launches0);
            report->precision_used = DT_PREC_FP64;
            report->ttm_x_launches = timer.count();
            report->ttm_x_ms = timer.total_ms();
            report->ttm_x_bytes = timer.bytes();
        }
    });
}

}  // extern "C"
