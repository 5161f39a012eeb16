// Sparse Tucker hot path: SpTensor construction with one mode-sorted copy of
// the nonzeros per mode, the TTMc (row-wise Kronecker accumulation of
// template/function/sp_tensor.tpp:288-417), its two contractions ttmc_mTR /
// ttmc_mTL (sp_tensor.tpp:236-365), and the sparse HOOI power sweep
// (template/algorithm/sp_tucker/sp_hooi_als.tpp:48-118).
//
// 3-way tensors (the configured workload) use a fibre-factored layout.  For
// mode n with other modes F (the "fibre" mode) and E, the nonzeros of row i_n
// are grouped by i_F, and
//     Y_(n)(i_n, :) = sum_{fibres f of the row} U_F(i_F(f), :) (x) w_f,
//     w_f = sum_{nonzeros e of f} v_e U_E(i_E(e), :),
// which costs R_E FMAs per nonzero and R_F R_E per fibre instead of R_F R_E per
// nonzero.  The outer products run on the FP64 tensor cores (mma.sync m8n8k4):
// four fibres form the K = 4 slice of one step.  Other orders use a row kernel
// (one warp per chunk of a row).
//
// Long rows are cut into pieces that write partial rows; a second kernel sums
// them in a fixed order, so the output is deterministic and needs no
// floating-point atomics.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dt_kernels.cuh"
#include "dt_sparse.cuh"

namespace dt {
namespace {

constexpr int64_t CHUNK = 512;
constexpr int FIB_CHUNK = 8;
constexpr int64_t TASK_PACK_GRP = 128;
constexpr int64_t TASK_PIECE_BATCHES = 64;

}  // namespace
}  // namespace dt

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
// TTMc row kernel (orders other than 3).  One warp per chunk.  Lane l owns
// Kronecker entries p = l + 32 q (q < PL); per nonzero it multiplies the
// value by the other factors' entries at its p.
// ---------------------------------------------------------------------------
template <int PL>
__global__ void __launch_bounds__(256) ttmc_rows_kernel(
    const int32_t *__restrict__ other, const double *__restrict__ val, int64_t nnz, int nother,
    const int64_t *__restrict__ rowptr, const int32_t *__restrict__ chunk_row,
    const int64_t *__restrict__ chunk_beg, const int32_t *__restrict__ chunk_slot,
    int64_t nchunks, FactorSet f, int P, double *__restrict__ Yc, double *__restrict__ Ypart) {
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
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
                int32_t ix[MAXD - 1];
#pragma unroll
                for (int d = 0; d < MAXD - 1; d++) ix[d] = __shfl_sync(0xffffffffu, myidx[d], j);
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
        const int32_t slot = chunk_slot[c];
        double *dst = slot < 0 ? Yc + (int64_t)k * P : Ypart + (int64_t)slot * P;
#pragma unroll
        for (int q = 0; q < PL; q++) {
            const int p = lane + 32 * q;
            if (p < P) dst[p] = acc[q];
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core fragment helper (mma.sync m8n8k4 .f64).  Fragments: A[g][t]
// and B[t][g] with g = lane / 4, t = lane % 4; the 8 x 8 result D[g][2t + {0,1}].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sp_dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// 3-way fibre TTMc.  The Kronecker index is p = p_lo + R_lo p_hi over the two
// other modes (lower mode fastest, sp_tensor.tpp:367-417); the warp keeps the
// current row as TR x TC tiles of 8 x 8 with rows = p_hi and columns = p_lo,
// so each lane's two accumulators of a tile are adjacent in memory.
//
// Layout: every row's (sub-)fibres, longest first, padded to a multiple of 4
// with empty fibres; four consecutive fibres form a group, the K = 4 slice of
// one mma.sync step.  Lane (g, t) takes fibre t of the group: it sums
// w = sum_e v_e U_E(i_E(e), g + 8 j) over its fibre's nonzeros and reads
// U_F(i_F, g + 8 j) -- exactly its A / B fragment elements -- so the group's
// four outer products are TF x TE mma.sync steps with no redundant FMAs.
// FLO: the fibre mode is the lower of the two (columns are p_F), else the
// higher (rows are p_F).
//
// Pipeline (one warp per task = a run of batches; a batch is at most FB_GRP
// groups and FB_NZ nonzeros, precomputed):
//  * batch b + 2: fibre indices / offsets, nonzero indices / values and the
//    groups' rows are loaded into registers (coalesced, one lane per item);
//  * batch b + 1: its U_E rows (one per nonzero) and U_F rows (one per fibre)
//    are copied by 16-byte cp.async into the warp's shared stage (the values
//    and offsets by plain stores);
//  * batch b: the fibre sums and the mma.sync steps read only shared memory.
// A row is written when its last group is done (rows of a task are whole,
// except pieces of long rows, which write a partial row at the task's end).
// ---------------------------------------------------------------------------
constexpr int FB_NZ = 32;
constexpr int FB_GRP = 4;
constexpr int FB_SLOTS = 4 * FB_GRP;
// One lane per staged nonzero and per fibre slot.
static_assert(FB_NZ <= 32 && FB_SLOTS <= 32 && 4 * FIB_CHUNK <= FB_NZ, "batch limits");
constexpr int FB_ROW_END = 1 << 8;  // grp_aux: the group is the last of its row

// A staged factor row of up to 8 T entries has a pitch of 8 T doubles.  Four
// rows read by one fragment load (8 consecutive doubles each) start in the
// same bank when the pitch is 16 or 32 doubles, so column c of row j is stored
// at c ^ fb_swz(j): rows alternate between the two 64-byte halves of a bank
// cycle (pitch 16) or its four 64-byte quarters (pitch 32).  Pitches 8 and 24
// alternate by themselves.
__host__ __device__ constexpr int fb_pitch(int T) { return 8 * T; }
__device__ __forceinline__ int fb_swz(int row, int pitch) {
    return pitch == 16 ? (row & 1) << 3 : pitch == 32 ? (row & 3) << 3 : 0;
}

template <int TF, int TE>
struct FbStage {
    static constexpr int PE = fb_pitch(TE), PF = fb_pitch(TF);
    static constexpr int DOUBLES = FB_NZ * PE + FB_SLOTS * PF + FB_NZ;
    static constexpr int INTS = FB_SLOTS + 1 + 2 * FB_GRP;
    static constexpr int BYTES = DOUBLES * 8 + ((INTS * 4 + 15) & ~15);
    static constexpr int WARP_BYTES = 2 * BYTES;
};

__device__ __forceinline__ void sp_cp16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void sp_cp8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void sp_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void sp_cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

struct FbMeta {
    int g0, ng, nz0, nzn;
    int fidx, fofs, grow, gaux;
    int idx;
    double v;
};

// Registers of batch b: lane l holds fibre slot l (index, offset into the
// batch's nonzeros), nonzero l (index, value) and group l's row and aux word
// (longest fibre | FB_ROW_END when the group is the last of its row).
__device__ __forceinline__ void fb_load_meta(FbMeta &m, int b, int lane,
                                             const int2 *__restrict__ bt,
                                             const int32_t *__restrict__ grp_row,
                                             const int32_t *__restrict__ grp_aux,
                                             const int32_t *__restrict__ fib_idx,
                                             const int32_t *__restrict__ fib_ptr,
                                             const int32_t *__restrict__ e_idx,
                                             const double *__restrict__ e_val) {
    const int2 c = bt[b], d = bt[b + 1];
    m.g0 = c.x;
    m.ng = d.x - c.x;
    m.nz0 = c.y;
    m.nzn = d.y - c.y;
    const bool sv = lane < 4 * m.ng;
    m.fidx = sv ? fib_idx[4 * m.g0 + lane] : 0;
    m.fofs = sv ? fib_ptr[4 * m.g0 + lane] - m.nz0 : 0;
    m.grow = lane < m.ng ? grp_row[m.g0 + lane] : 0;
    m.gaux = lane < m.ng ? grp_aux[m.g0 + lane] : 0;
    const bool a = lane < m.nzn;
    m.idx = a ? e_idx[m.nz0 + lane] : 0;
    m.v = a ? e_val[m.nz0 + lane] : 0.0;
}

__host__ __device__ constexpr int fb_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Copies n <= 32 rows of the transposed factor U (R <= RMAX doubles each; the
// index of row j is held by lane j) into dst rows of RMAX doubles, swizzled
// (fb_swz).  Lane l copies piece l % PPR of row l / PPR (+ 32 / PPR per step),
// PPR a power of two: 16-byte pieces when R is even and U 16-byte aligned,
// else 8-byte ones.
template <int RMAX>
__device__ __forceinline__ void fb_stage_rows(double *dst, const double *__restrict__ U, int R,
                                              int n, int ridx, int lane) {
    constexpr int pitch = RMAX;
    if ((R & 1) == 0 && (reinterpret_cast<uintptr_t>(U) & 15) == 0) {
        constexpr int PPR = fb_pow2(RMAX / 2), RPI = 32 / PPR;
        const int rem = lane % PPR, jl = lane / PPR;
        const bool okp = 2 * rem < R;
        for (int j0 = 0; j0 < n; j0 += RPI) {
            const int j = j0 + jl;
            const int i = __shfl_sync(0xffffffffu, ridx, j & 31);
            if (j < n && okp)
                sp_cp16(dst + j * pitch + ((2 * rem) ^ fb_swz(j, pitch)),
                        U + (int64_t)i * R + 2 * rem);
        }
    } else {
        constexpr int PPR = fb_pow2(RMAX), RPI = 32 / PPR;
        const int rem = lane % PPR, jl = lane / PPR;
        const bool okp = rem < R;
        for (int j0 = 0; j0 < n; j0 += RPI) {
            const int j = j0 + jl;
            const int i = __shfl_sync(0xffffffffu, ridx, j & 31);
            if (j < n && okp)
                sp_cp8(dst + j * pitch + (rem ^ fb_swz(j, pitch)), U + (int64_t)i * R + rem);
        }
    }
}

template <int TF, int TE, bool FLO>
__global__ void __launch_bounds__(256, 2) ttmc3f_kernel(
    const int4 *__restrict__ tasks, int64_t ntasks, const int2 *__restrict__ bt,
    const int32_t *__restrict__ grp_row, const int32_t *__restrict__ grp_aux,
    const int32_t *__restrict__ fib_idx, const int32_t *__restrict__ fib_ptr,
    const int32_t *__restrict__ e_idx, const double *__restrict__ e_val,
    const double *__restrict__ UF, int RF, const double *__restrict__ UE, int RE,
    double *__restrict__ Yc, double *__restrict__ Ypart, int *__restrict__ next_task) {
    using S = FbStage<TF, TE>;
    constexpr int TR = FLO ? TE : TF, TC = FLO ? TF : TE;
    extern __shared__ __align__(16) unsigned char fb_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = lane >> 2, t4 = lane & 3;
    const int nwarp_blk = blockDim.x >> 5;
    unsigned char *wsm = fb_smem + (size_t)wib * S::WARP_BYTES;
    const int64_t gw = (int64_t)blockIdx.x * nwarp_blk + wib;
    const int64_t nw = (int64_t)gridDim.x * nwarp_blk;
    const int P = RF * RE;
    const int Rlo = FLO ? RF : RE, Rhi = FLO ? RE : RF;
    constexpr int pe = S::PE, pf = S::PF;
    bool okF[TF], okE[TE];
#pragma unroll
    for (int j = 0; j < TF; j++) okF[j] = g + 8 * j < RF;
#pragma unroll
    for (int j = 0; j < TE; j++) okE[j] = g + 8 * j < RE;
    // This lane's two output entries of tile (r, c) in a row: p = pl + Rlo ph
    // (-1: outside the row).
    int off[TR][TC];
#pragma unroll
    for (int r = 0; r < TR; r++)
#pragma unroll
        for (int c = 0; c < TC; c++) {
            const int ph = 8 * r + g, pl = 8 * c + 2 * t4;
            off[r][c] = (ph < Rhi && pl < Rlo) ? pl + Rlo * ph : -1;
        }
    const bool pair = (Rlo & 1) == 0;

    auto ue_of = [&](int buf) { return reinterpret_cast<double *>(wsm + buf * S::BYTES); };
    auto uf_of = [&](int buf) { return ue_of(buf) + FB_NZ * S::PE; };
    auto vv_of = [&](int buf) { return uf_of(buf) + FB_SLOTS * S::PF; };
    auto fo_of = [&](int buf) {
        return reinterpret_cast<int *>(wsm + buf * S::BYTES + S::DOUBLES * 8);
    };

    auto stage = [&](const FbMeta &m, int buf) {
        double *vv = vv_of(buf);
        int *fo = fo_of(buf);
        int *gr = fo + FB_SLOTS + 1;
        if (lane < FB_NZ) vv[lane] = m.v;
        if (lane < 4 * m.ng) fo[lane] = m.fofs;
        if (lane == 0) fo[4 * m.ng] = m.nzn;
        if (lane < m.ng) {
            gr[lane] = m.grow;
            gr[FB_GRP + lane] = m.gaux;
        }
        fb_stage_rows<8 * TE>(ue_of(buf), UE, RE, m.nzn, m.idx, lane);
        fb_stage_rows<8 * TF>(uf_of(buf), UF, RF, 4 * m.ng, m.fidx, lane);
        sp_cp_commit();
    };

    double acc[TR][TC][2];
#pragma unroll
    for (int r = 0; r < TR; r++)
#pragma unroll
        for (int c = 0; c < TC; c++) acc[r][c][0] = acc[r][c][1] = 0.0;

    // The first task of each warp is its own; later ones come from a counter
    // (dynamic balance over the largest-first task list).
    for (int64_t tk = gw; tk < ntasks;) {
        const int4 task = tasks[tk];
        const int b0 = task.x, b1 = task.y, slot = task.z;
        FbMeta m;
        fb_load_meta(m, b0, lane, bt, grp_row, grp_aux, fib_idx, fib_ptr, e_idx, e_val);
        stage(m, 0);
        int ng_cur = m.ng, ng_next = 0;
        if (b0 + 1 < b1)
            fb_load_meta(m, b0 + 1, lane, bt, grp_row, grp_aux, fib_idx, fib_ptr, e_idx, e_val);
        for (int b = b0; b < b1; b++) {
            const int buf = (b - b0) & 1;
            if (b + 1 < b1) {
                stage(m, buf ^ 1);
                ng_next = m.ng;
                if (b + 2 < b1)
                    fb_load_meta(m, b + 2, lane, bt, grp_row, grp_aux, fib_idx, fib_ptr, e_idx,
                                 e_val);
                sp_cp_wait<1>();
            } else {
                sp_cp_wait<0>();
            }
            __syncwarp();
            const double *ue = ue_of(buf), *uf = uf_of(buf), *vv = vv_of(buf);
            const int *fo = fo_of(buf);
            const int *gr = fo + FB_SLOTS + 1;
#pragma unroll
            for (int j = 0; j < FB_GRP; j++) {
                if (j >= ng_cur) break;
                const int s = 4 * j + t4;
                const int beg = fo[s], len = fo[s + 1] - beg;
                const int aux = gr[FB_GRP + j];
                const int mx = aux & (FB_ROW_END - 1);
                double w[TE];
#pragma unroll
                for (int k = 0; k < TE; k++) w[k] = 0.0;
                for (int q = 0; q < mx; q++) {
                    if (q < len) {
                        const int r = beg + q;
                        const double v = vv[r];
                        const double *rw = ue + r * pe;
                        const int sw = fb_swz(r, pe);
#pragma unroll
                        for (int k = 0; k < TE; k++)
                            if (okE[k]) w[k] = fma(v, rw[(g + 8 * k) ^ sw], w[k]);
                    }
                }
                double u[TF];
                const int swf = fb_swz(s, pf);
#pragma unroll
                for (int k = 0; k < TF; k++)
                    u[k] = (okF[k] && len > 0) ? uf[s * pf + ((g + 8 * k) ^ swf)] : 0.0;
#pragma unroll
                for (int r = 0; r < TR; r++)
#pragma unroll
                    for (int c = 0; c < TC; c++)
                        sp_dmma(acc[r][c][0], acc[r][c][1], FLO ? w[r] : u[r], FLO ? u[c] : w[c]);
                if ((aux & FB_ROW_END) || (b == b1 - 1 && j == ng_cur - 1)) {
                    double *dst = slot >= 0 ? Ypart + (int64_t)slot * P : Yc + (int64_t)gr[j] * P;
#pragma unroll
                    for (int r = 0; r < TR; r++)
#pragma unroll
                        for (int c = 0; c < TC; c++) {
                            const int o = off[r][c];
                            if (o >= 0) {
                                if (pair) {
                                    *reinterpret_cast<double2 *>(dst + o) =
                                        make_double2(acc[r][c][0], acc[r][c][1]);
                                } else {
                                    dst[o] = acc[r][c][0];
                                    if (8 * c + 2 * t4 + 1 < Rlo) dst[o + 1] = acc[r][c][1];
                                }
                            }
                            acc[r][c][0] = acc[r][c][1] = 0.0;
                        }
                }
            }
            __syncwarp();
            ng_cur = ng_next;
        }
        int nt = 0;
        if (lane == 0) nt = atomicAdd(next_task, 1);
        tk = nw + __shfl_sync(0xffffffffu, nt, 0);
    }
}

// Fibre TTMc for other-mode ranks above 32 (P <= 1024): lane l owns Kronecker
// entries p = l + 32 q, q < PL; per fibre it accumulates w at its p_E, then
// one FMA with U_F at its p_F.  Same task / batch / group structure.
template <int PL, bool FLO>
__global__ void __launch_bounds__(256) ttmc3f_wide_kernel(
    const int4 *__restrict__ tasks, int64_t ntasks, const int2 *__restrict__ bt,
    const int32_t *__restrict__ grp_row, const int32_t *__restrict__ grp_aux,
    const int32_t *__restrict__ fib_idx, const int32_t *__restrict__ fib_ptr,
    const int32_t *__restrict__ e_idx, const double *__restrict__ e_val,
    const double *__restrict__ UF, int RF, const double *__restrict__ UE, int RE,
    double *__restrict__ Yc, double *__restrict__ Ypart) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int P = RF * RE;
    const int Rlo = FLO ? RF : RE;
    int pF[PL], pE[PL];
#pragma unroll
    for (int q = 0; q < PL; q++) {
        const int p = min(lane + 32 * q, P - 1);
        const int lo = p % Rlo, hi = p / Rlo;
        pF[q] = FLO ? lo : hi;
        pE[q] = FLO ? hi : lo;
    }
    double acc[PL];
#pragma unroll
    for (int q = 0; q < PL; q++) acc[q] = 0.0;
    for (int64_t tk = gw; tk < ntasks; tk += nw) {
        const int4 task = tasks[tk];
        const int gbeg = bt[task.x].x, gend = bt[task.y].x, slot = task.z;
        for (int gq = gbeg; gq < gend; gq++) {
            for (int f = 4 * gq; f < 4 * gq + 4; f++) {
                const int fi = fib_idx[f], b = fib_ptr[f], e = fib_ptr[f + 1];
                if (b == e) continue;
                double w[PL];
#pragma unroll
                for (int q = 0; q < PL; q++) w[q] = 0.0;
                for (int j = b; j < e; j++) {
                    const double v = __ldg(e_val + j);
                    const double *u = UE + (int64_t)__ldg(e_idx + j) * RE;
#pragma unroll
                    for (int q = 0; q < PL; q++) w[q] = fma(v, __ldg(u + pE[q]), w[q]);
                }
                const double *u = UF + (int64_t)fi * RF;
#pragma unroll
                for (int q = 0; q < PL; q++) acc[q] = fma(__ldg(u + pF[q]), w[q], acc[q]);
            }
            if ((grp_aux[gq] & FB_ROW_END) || gq == gend - 1) {
                double *dst = slot >= 0 ? Ypart + (int64_t)slot * P : Yc + (int64_t)grp_row[gq] * P;
#pragma unroll
                for (int q = 0; q < PL; q++) {
                    if (lane + 32 * q < P) dst[lane + 32 * q] = acc[q];
                    acc[q] = 0.0;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Yc[row] = sum of its partial rows.  One CTA of 4 x 256 threads per row:
// thread (s, x) sums partials c = s, s + 4, ... of entry p = x (+ 256 ...)
// into four accumulators (c mod 16), so 16 independent loads are in flight;
// the 4 x 4 accumulators are then added in a fixed order (deterministic).
// ---------------------------------------------------------------------------
constexpr int COMB_SPLIT = 4;
constexpr int COMB_SEG = 16;

// First level of the fibre path's combine: seg_out[g] = the sum, in order, of
// the tseg_count[g] partial rows from slot tseg_first[g] (at most COMB_SEG;
// four accumulators, fixed order).
__global__ void __launch_bounds__(256) sum_segments_kernel(
    const double *__restrict__ Ypart, const int32_t *__restrict__ seg_first,
    const int32_t *__restrict__ seg_count, int64_t nseg, int P, double *__restrict__ seg_out) {
    for (int64_t g = blockIdx.x; g < nseg; g += gridDim.x) {
        const int64_t f = seg_first[g];
        const int cnt = seg_count[g];
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int j = 0; j < COMB_SEG; j++)
                if (j < cnt) a[j & 3] += Ypart[(f + j) * P + p];
            seg_out[g * P + p] = (a[0] + a[1]) + (a[2] + a[3]);
        }
    }
}
__global__ void __launch_bounds__(1024) combine_partials_kernel(
    const double *__restrict__ Ypart, const int32_t *__restrict__ multi_row,
    const int32_t *__restrict__ multi_first, const int32_t *__restrict__ multi_count,
    int64_t nmulti, int P, double *__restrict__ Yc) {
    __shared__ double red[COMB_SPLIT][256];
    const int s = threadIdx.x >> 8, x = threadIdx.x & 255;
    for (int64_t m = blockIdx.x; m < nmulti; m += gridDim.x) {
        const int32_t k = multi_row[m];
        const int64_t first = multi_first[m];
        const int cnt = multi_count[m];
        for (int p0 = 0; p0 < P; p0 += 256) {
            const int p = p0 + x;
            double a[4] = {0.0, 0.0, 0.0, 0.0};
            if (p < P) {
                const double *src = Ypart + (first + s) * P + p;
                int c = s;
                for (; c + 3 * COMB_SPLIT < cnt; c += 4 * COMB_SPLIT) {
#pragma unroll
                    for (int j = 0; j < 4; j++) a[j] += src[(int64_t)j * COMB_SPLIT * P];
                    src += (int64_t)4 * COMB_SPLIT * P;
                }
#pragma unroll
                for (int j = 0; j < 3; j++)
                    if (c + j * COMB_SPLIT < cnt) a[j] += src[(int64_t)j * COMB_SPLIT * P];
            }
            red[s][x] = (a[0] + a[1]) + (a[2] + a[3]);
            __syncthreads();
            if (s == 0 && p < P)
                Yc[(int64_t)k * P + p] = (red[0][x] + red[1][x]) + (red[2][x] + red[3][x]);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// ttmc_mTL / ttmc_mTR on the FP64 tensor-core path (sp_dmma above).  Staged
// shared operands use a pitch of 4 (mod 16) doubles so a half-warp's fragment
// loads hit distinct banks.
// ---------------------------------------------------------------------------

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
        // Eight k-steps of Y loads are issued before their MMAs.
        for (int k0 = 0; k0 < ksteps; k0 += 8) {
            double av[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int p = 4 * (k0 + u) + t;
                av[u] = (okr && k0 + u < ksteps && p < P) ? y[p] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                if (k0 + u >= ksteps) break;
                const int p = 4 * (k0 + u) + t;
#pragma unroll
                for (int j = 0; j < NTL; j++) {
                    const int r = 8 * j + g;
                    const double b =
                        LSM ? Ls[p * LDL + r]
                            : ((p < P && r < Rn) ? __ldg(L + p + (int64_t)P * r) : 0.0);
                    sp_dmma(acc[j][0], acc[j][1], av[u], b);
                }
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
            // Four k-steps of Yc loads are issued before their MMAs, so 4 MG
            // loads per lane are in flight.
            for (int ks0 = 0; ks0 < ks_end; ks0 += 4) {
                double av[4][MG], bv[4][NTL];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int bl = 4 * (ks0 + u) + t;
                    const int64_t k = kb + bl;
                    const bool okk = bl < kn;
#pragma unroll
                    for (int j = 0; j < NTL; j++) bv[u][j] = okk ? Us[bl * LDU + 8 * j + g] : 0.0;
#pragma unroll
                    for (int m = 0; m < MG; m++) {
                        const int mt = mbase + w + 8 * m;
                        const int p = 8 * mt + g;
                        av[u][m] = (okk && mt < ptiles && p < P) ? Yc[k * P + p] : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int m = 0; m < MG; m++)
#pragma unroll
                        for (int j = 0; j < NTL; j++)
                            sp_dmma(acc[m][j][0], acc[m][j][1], av[u][m], bv[u][j]);
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

// out[e] = sum_b part[b * n + e]: 64 outputs per CTA, 4 threads per output
// each summing every 4th block into 4 accumulators (16 loads in flight), then
// a fixed-order add (deterministic).
__global__ void __launch_bounds__(256) sum_blocks_kernel(const double *__restrict__ part,
                                                         int nblk, int64_t n,
                                                         double *__restrict__ out) {
    __shared__ double red[4][64];
    const int s = threadIdx.x >> 6, o = threadIdx.x & 63;
    for (int64_t e0 = (int64_t)blockIdx.x * 64; e0 < n; e0 += (int64_t)gridDim.x * 64) {
        const int64_t e = e0 + o;
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

int64_t kron_len(const int64_t *R, int ndim, int mode) {
    int64_t P = 1;
    for (int m = 0; m < ndim; m++)
        if (m != mode) P *= R[m];
    return P;
}

// Uploads a host vector into a device buffer (at least 8 bytes).
template <class T>
void upload(dt_ctx *ctx, DevMem &dst, const std::vector<T> &src) {
    const size_t bytes = src.size() * sizeof(T);
    dst.alloc(ctx, std::max<size_t>(bytes, 8));
    if (bytes)
        DT_CUDA(cudaMemcpyAsync(dst.get(), src.data(), bytes, cudaMemcpyHostToDevice,
                                ctx->stream));
}

int index_bits(int64_t extent) {
    int bits = 1;
    while ((int64_t(1) << bits) < extent) bits++;
    return bits;
}

// Row-kernel layout: stable radix sort of (row index, nonzero id), the other
// modes' indices and the values gathered into that order, and the chunk list.
void build_mode_rows(dt_ctx *ctx, dt_sptensor *sp, int n, const std::vector<DevMem> &idx32,
                     const double *vals_dev) {
    ModeCopy &mc = sp->modes[n];
    const int64_t nnz = sp->nnz;
    const int nd = sp->ndim;
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceil_div(nnz, 256), 8 * ctx->num_sms));
    DevMem ids(ctx, nnz * sizeof(int32_t)), keys_out(ctx, nnz * sizeof(int32_t)),
        perm(ctx, nnz * sizeof(int32_t));
    DT_LAUNCH(ctx, iota_kernel, blocks, 256, 0, ids.as<int32_t>(), nnz);
    const int bits = index_bits(sp->shape[n]);
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
    upload(ctx, mc.rows, rows);
    upload(ctx, mc.rowptr, rowptr);
    upload(ctx, mc.chunk_row, crow);
    upload(ctx, mc.chunk_beg, cbeg);
    upload(ctx, mc.chunk_slot, cslot);
    upload(ctx, mc.multi_row, mrow);
    upload(ctx, mc.multi_first, mfirst);
    upload(ctx, mc.multi_count, mcount);
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
}

__global__ void fibre_key_kernel(const int32_t *__restrict__ in, const int32_t *__restrict__ iF,
                                 int bitsF, int64_t n, uint64_t *__restrict__ key) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x)
        key[e] = ((uint64_t)(uint32_t)in[e] << bitsF) | (uint32_t)iF[e];
}

// Fibre layout of a 3-way tensor for mode n.  Both other modes are tried as
// the fibre mode F (radix sort of the 64-bit key (i_n, i_F) with the nonzero
// ids); the one giving fewer fibres is kept.  On the host: fibres longer than
// FIB_CHUNK nonzeros are cut into sub-fibres, a row's (sub-)fibres are ordered
// by length, longest first (stable), and the nonzeros are permuted to follow;
// the task list packs whole rows and cuts long rows into pieces.
void build_mode_fibre(dt_ctx *ctx, dt_sptensor *sp, int n, const std::vector<DevMem> &idx32,
                      const double *vals_dev) {
    ModeCopy &mc = sp->modes[n];
    const int64_t nnz = sp->nnz;
    int oth[2], d = 0;
    for (int m = 0; m < 3; m++)
        if (m != n) oth[d++] = m;
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceil_div(nnz, 256), 8 * ctx->num_sms));
    const int bits_n = index_bits(sp->shape[n]);
    DevMem key(ctx, nnz * sizeof(uint64_t)), key_s(ctx, nnz * sizeof(uint64_t)),
        ids(ctx, nnz * sizeof(int32_t)), ids_s(ctx, nnz * sizeof(int32_t));
    std::vector<uint64_t> hkey((size_t)nnz), best_key;
    std::vector<int32_t> best_ids((size_t)nnz);
    int64_t best_fib = -1;
    int best_F = -1, best_bits = 0;
    DevMem tmp;
    size_t tmp_have = 0;
    for (int c = 0; c < 2; c++) {
        const int F = oth[c];
        const int bits_F = index_bits(sp->shape[F]);
        DT_LAUNCH(ctx, fibre_key_kernel, blocks, 256, 0, idx32[n].as<int32_t>(),
                  idx32[F].as<int32_t>(), bits_F, nnz, key.as<uint64_t>());
        DT_LAUNCH(ctx, iota_kernel, blocks, 256, 0, ids.as<int32_t>(), nnz);
        size_t tmp_bytes = 0;
        DT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.as<uint64_t>(),
                                                key_s.as<uint64_t>(), ids.as<int32_t>(),
                                                ids_s.as<int32_t>(), (int)nnz, 0,
                                                bits_n + bits_F, ctx->stream));
        if (tmp_bytes > tmp_have) {
            tmp.alloc(ctx, tmp_bytes);
            tmp_have = tmp_bytes;
        }
        DT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, key.as<uint64_t>(),
                                                key_s.as<uint64_t>(), ids.as<int32_t>(),
                                                ids_s.as<int32_t>(), (int)nnz, 0,
                                                bits_n + bits_F, ctx->stream));
        ctx->launches += 1;
        DT_CUDA(cudaMemcpyAsync(hkey.data(), key_s.get(), nnz * sizeof(uint64_t),
                                cudaMemcpyDeviceToHost, ctx->stream));
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
        int64_t fib = 0;
        for (int64_t e = 0; e < nnz; e++) fib += (e == 0 || hkey[e] != hkey[e - 1]);
        if (best_fib < 0 || fib < best_fib) {
            best_fib = fib;
            best_F = F;
            best_bits = bits_F;
            best_key.swap(hkey);
            if (hkey.size() != (size_t)nnz) hkey.resize((size_t)nnz);
            DT_CUDA(cudaMemcpyAsync(best_ids.data(), ids_s.get(), nnz * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, ctx->stream));
            DT_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    }
    hkey.clear();
    hkey.shrink_to_fit();
    mc.fmode = best_F;
    const int E = oth[0] == best_F ? oth[1] : oth[0];
    const uint64_t fmask = (uint64_t(1) << best_bits) - 1;

    // Rows, (sub-)fibres in length order padded to groups of four, and the
    // permuted nonzero order.
    struct Fib {
        int64_t beg;
        int32_t len, idx;
    };
    std::vector<int32_t> rows, row_grp, grp_row, grp_aux, fib_idx, fib_ptr, order;
    fib_idx.reserve((size_t)best_fib * 5 / 4 + 16);
    fib_ptr.reserve((size_t)best_fib * 5 / 4 + 17);
    order.reserve((size_t)nnz);
    std::vector<Fib> rf;
    int64_t e = 0;
    while (e < nnz) {
        const uint64_t r = best_key[e] >> best_bits;
        rf.clear();
        while (e < nnz && (best_key[e] >> best_bits) == r) {
            const uint64_t kf = best_key[e];
            const int64_t b = e;
            while (e < nnz && best_key[e] == kf) e++;
            for (int64_t s = b; s < e; s += FIB_CHUNK)
                rf.push_back({s, (int32_t)std::min<int64_t>(FIB_CHUNK, e - s),
                              (int32_t)(kf & fmask)});
        }
        std::stable_sort(rf.begin(), rf.end(),
                         [](const Fib &a, const Fib &b) { return a.len > b.len; });
        while (rf.size() % 4) rf.push_back({0, 0, 0});
        const int32_t k = (int32_t)rows.size();
        rows.push_back((int32_t)r);
        row_grp.push_back((int32_t)(fib_idx.size() / 4));
        for (const Fib &f : rf) {
            fib_idx.push_back(f.idx);
            fib_ptr.push_back((int32_t)order.size());
            for (int32_t j = 0; j < f.len; j++) order.push_back(best_ids[f.beg + j]);
        }
        for (size_t q = 0; q < rf.size() / 4; q++) {
            grp_row.push_back(k);
            int32_t mx = 0;
            for (int t = 0; t < 4; t++) mx = std::max(mx, rf[4 * q + t].len);
            grp_aux.push_back(mx | (q + 1 == rf.size() / 4 ? FB_ROW_END : 0));
        }
    }
    const int32_t ngroups = (int32_t)(fib_idx.size() / 4);
    row_grp.push_back(ngroups);
    fib_ptr.push_back((int32_t)order.size());
    best_key.clear();
    best_key.shrink_to_fit();
    mc.nrows = (int64_t)rows.size();
    mc.nfib = (int64_t)fib_idx.size();

    // Tasks over groups: packs of whole rows up to TASK_PACK_GRP groups; longer
    // rows in pieces of TASK_PIECE_BATCHES batches writing partial rows.  Each task
    // is cut into batches of at most FB_GRP groups and FB_NZ nonzeros (a group
    // holds at most 4 FIB_CHUNK <= FB_NZ).  Cost estimate for the
    // largest-first order: nonzeros + 16 per group.
    auto gnz = [&](int32_t q) { return fib_ptr[4 * q + 4] - fib_ptr[4 * q]; };
    std::vector<int2> bt;
    struct Task {
        int4 t;
        int64_t cost;
    };
    std::vector<Task> tasks;
    std::vector<int32_t> tmrow, tmfirst, tmcount, tsfirst, tscount;
    int64_t tslots = 0;
    // Batches of the groups [q0, q1), appended to bt; returns how many.
    auto make_batches = [&](int32_t q0, int32_t q1) {
        int32_t nb = 0, q = q0;
        while (q < q1) {
            bt.push_back(make_int2(q, fib_ptr[4 * q]));
            nb++;
            int32_t nz = 0, cnt = 0;
            while (q < q1 && cnt < FB_GRP && nz + gnz(q) <= FB_NZ) {
                nz += gnz(q);
                cnt++;
                q++;
            }
        }
        return nb;
    };
    // A warp spends about the same time on every batch, so a task's cost is
    // its batch count.
    auto add_pack = [&](int32_t q0, int32_t q1) {
        const int32_t b0 = (int32_t)bt.size();
        const int32_t nb = make_batches(q0, q1);
        tasks.push_back({make_int4(b0, b0 + nb, -1, 0), nb});
    };
    {
        int32_t pack_beg = -1;
        for (int64_t k = 0; k < mc.nrows; k++) {
            const int32_t b = row_grp[k], c = row_grp[k + 1] - b;
            if (c > TASK_PACK_GRP) {
                if (pack_beg >= 0) add_pack(pack_beg, b);
                pack_beg = -1;
                // A long row: its batches in pieces of at most TASK_PIECE_BATCHES.
                const int32_t b0 = (int32_t)bt.size();
                const int32_t nb = make_batches(b, b + c);
                const int32_t np = (nb + (int32_t)TASK_PIECE_BATCHES - 1) / (int32_t)TASK_PIECE_BATCHES;
                if (np > 1) {
                    tmrow.push_back((int32_t)k);
                    tmfirst.push_back((int32_t)tsfirst.size());
                    for (int32_t q = 0; q < np; q += COMB_SEG) {
                        tsfirst.push_back((int32_t)tslots + q);
                        tscount.push_back(std::min<int32_t>(COMB_SEG, np - q));
                    }
                    tmcount.push_back((int32_t)tsfirst.size() - tmfirst.back());
                }
                for (int32_t j = 0; j < np; j++) {
                    const int32_t x0 = b0 + j * (int32_t)TASK_PIECE_BATCHES;
                    const int32_t x1 = std::min(b0 + nb, x0 + (int32_t)TASK_PIECE_BATCHES);
                    tasks.push_back({make_int4(x0, x1, np > 1 ? (int32_t)(tslots + j) : -1, 0),
                                     x1 - x0});
                }
                if (np > 1) tslots += np;
                continue;
            }
            if (pack_beg >= 0 && b + c - pack_beg > TASK_PACK_GRP) {
                add_pack(pack_beg, b);
                pack_beg = -1;
            }
            if (pack_beg < 0) pack_beg = b;
        }
        if (pack_beg >= 0) add_pack(pack_beg, ngroups);
        bt.push_back(make_int2(ngroups, fib_ptr[4 * ngroups]));
        std::stable_sort(tasks.begin(), tasks.end(),
                         [](const Task &a, const Task &b) { return a.cost > b.cost; });
    }
    std::vector<int4> tv(tasks.size());
    for (size_t i = 0; i < tasks.size(); i++) tv[i] = tasks[i].t;
    mc.ntasks = (int64_t)tv.size();
    mc.nbatch = (int64_t)bt.size() - 1;
    mc.tslots = tslots;
    mc.tmulti = (int64_t)tmrow.size();
    mc.nseg = (int64_t)tsfirst.size();

    DevMem perm;
    upload(ctx, perm, order);
    mc.e_idx.alloc(ctx, nnz * sizeof(int32_t));
    mc.e_val.alloc(ctx, nnz * sizeof(double));
    DT_LAUNCH(ctx, gather_kernel<int32_t>, blocks, 256, 0, idx32[E].as<int32_t>(),
              perm.as<int32_t>(), nnz, mc.e_idx.as<int32_t>());
    DT_LAUNCH(ctx, gather_kernel<double>, blocks, 256, 0, vals_dev, perm.as<int32_t>(), nnz,
              mc.e_val.as<double>());
    upload(ctx, mc.rows, rows);
    upload(ctx, mc.grp_row, grp_row);
    upload(ctx, mc.grp_aux, grp_aux);
    upload(ctx, mc.fib_idx, fib_idx);
    upload(ctx, mc.fib_ptr, fib_ptr);
    upload(ctx, mc.batches, bt);
    upload(ctx, mc.tasks, tv);
    upload(ctx, mc.tmulti_row, tmrow);
    upload(ctx, mc.tmulti_first, tmfirst);
    upload(ctx, mc.tmulti_count, tmcount);
    upload(ctx, mc.tseg_first, tsfirst);
    upload(ctx, mc.tseg_count, tscount);
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
}

void build_mode(dt_ctx *ctx, dt_sptensor *sp, int n, const std::vector<DevMem> &idx32,
                const double *vals_dev) {
    if (sp->ndim == 3)
        build_mode_fibre(ctx, sp, n, idx32, vals_dev);
    else
        build_mode_rows(ctx, sp, n, idx32, vals_dev);
}

template <int PL>
void launch_rows(dt_ctx *ctx, const ModeCopy &mc, int nother, int64_t nnz, const FactorSet &f,
                 int P, double *Yc, double *Ypart) {
    const int64_t warps = mc.nchunks;
    const unsigned blocks =
        std::max(1u, std::min<unsigned>(ceil_div(warps, 8), 32u * (unsigned)ctx->num_sms));
    DT_LAUNCH(ctx, ttmc_rows_kernel<PL>, blocks, 256, 0, mc.other.as<int32_t>(),
              mc.val.as<double>(), nnz, nother, mc.rowptr.as<int64_t>(),
              mc.chunk_row.as<int32_t>(), mc.chunk_beg.as<int64_t>(),
              mc.chunk_slot.as<int32_t>(), mc.nchunks, f, P, Yc, Ypart);
}

template <int TF, int TE, bool FLO>
void launch_fib(dt_ctx *ctx, const ModeCopy &mc, const double *UF, int RF, const double *UE,
                int RE, double *Yc, double *Ypart) {
    using S = FbStage<TF, TE>;
    auto kern = ttmc3f_kernel<TF, TE, FLO>;
    // Two CTAs per SM when their stages fit in half of the 228 KB (1 KB of
    // each CTA's share is reserved), else one.
    int per_sm = 2, warps = std::min(8, (228 * 1024 / 2 - 1024) / S::WARP_BYTES);
    // An even warp count per CTA spreads warps evenly over the 4 schedulers.
    if (warps > 1 && warps < 8) warps &= ~1;
    if (warps < 1) {
        per_sm = 1;
        warps = std::max(1, std::min(8, (227 * 1024) / S::WARP_BYTES));
    }
    const size_t smem = (size_t)warps * S::WARP_BYTES;
    smem_limit(ctx, kern, smem);
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((mc.ntasks + warps - 1) / warps, (int64_t)per_sm * ctx->num_sms));
    DevMem next(ctx, sizeof(int));
    DT_CUDA(cudaMemsetAsync(next.get(), 0, sizeof(int), ctx->stream));
    DT_LAUNCH(ctx, kern, blocks, warps * 32, smem, mc.tasks.as<int4>(), mc.ntasks,
              mc.batches.as<int2>(), mc.grp_row.as<int32_t>(), mc.grp_aux.as<int32_t>(),
              mc.fib_idx.as<int32_t>(), mc.fib_ptr.as<int32_t>(), mc.e_idx.as<int32_t>(),
              mc.e_val.as<double>(), UF, RF, UE, RE, Yc, Ypart, next.as<int>());
}

template <int PL, bool FLO>
void launch_fib_wide(dt_ctx *ctx, const ModeCopy &mc, const double *UF, int RF, const double *UE,
                     int RE, double *Yc, double *Ypart) {
    auto kern = ttmc3f_wide_kernel<PL, FLO>;
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((mc.ntasks + 7) / 8, (int64_t)8 * ctx->num_sms));
    DT_LAUNCH(ctx, kern, blocks, 256, 0, mc.tasks.as<int4>(), mc.ntasks, mc.batches.as<int2>(),
              mc.grp_row.as<int32_t>(), mc.grp_aux.as<int32_t>(), mc.fib_idx.as<int32_t>(),
              mc.fib_ptr.as<int32_t>(), mc.e_idx.as<int32_t>(), mc.e_val.as<double>(), UF, RF,
              UE, RE, Yc, Ypart);
}

template <int TF, bool FLO>
void fib_dispatch_te(dt_ctx *ctx, const ModeCopy &mc, const double *UF, int RF, const double *UE,
                     int RE, double *Yc, double *Ypart) {
    switch ((RE + 7) / 8) {
        case 1: launch_fib<TF, 1, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
        case 2: launch_fib<TF, 2, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
        case 3: launch_fib<TF, 3, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
        default: launch_fib<TF, 4, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
    }
}

template <bool FLO>
void fib_dispatch(dt_ctx *ctx, const ModeCopy &mc, const double *UF, int RF, const double *UE,
                  int RE, double *Yc, double *Ypart) {
    if (RF > 32 || RE > 32) {
        const int PL = (RF * RE + 31) / 32;
        if (PL <= 8) launch_fib_wide<8, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart);
        else if (PL <= 16) launch_fib_wide<16, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart);
        else launch_fib_wide<32, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart);
        return;
    }
    switch ((RF + 7) / 8) {
        case 1: fib_dispatch_te<1, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
        case 2: fib_dispatch_te<2, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
        case 3: fib_dispatch_te<3, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
        default: fib_dispatch_te<4, FLO>(ctx, mc, UF, RF, UE, RE, Yc, Ypart); break;
    }
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
    if (nd == 3) {
        const int F = mc.fmode;
        int E = 0;
        for (int m = 0; m < 3; m++)
            if (m != mode && m != F) E = m;
        DevMem tpart(ctx, std::max<int64_t>(mc.tslots, 1) * P * sizeof(double));
        SummaryScope sc(ctx, "Function::ttmc()",
                        2.0 * ((double)sp->nnz * R[E] + (double)mc.nfib * R[F] * R[E]),
                        (double)sp->nnz * 12.0 + (double)mc.nfib * 8.0 +
                            (double)mc.nrows * P * 8.0);
        if (timer) timer->begin();
        if (F < E)
            fib_dispatch<true>(ctx, mc, Ut_dev[F], (int)R[F], Ut_dev[E], (int)R[E], Yc,
                               tpart.as<double>());
        else
            fib_dispatch<false>(ctx, mc, Ut_dev[F], (int)R[F], Ut_dev[E], (int)R[E], Yc,
                                tpart.as<double>());
        if (mc.tmulti > 0) {
            DevMem segs(ctx, (size_t)mc.nseg * P * sizeof(double));
            DT_LAUNCH(ctx, sum_segments_kernel,
                      (unsigned)std::min<int64_t>(mc.nseg, 65535), 256, 0, tpart.as<double>(),
                      mc.tseg_first.as<int32_t>(), mc.tseg_count.as<int32_t>(), mc.nseg, P,
                      segs.as<double>());
            const unsigned blocks = (unsigned)std::min<int64_t>(mc.tmulti, 65535);
            DT_LAUNCH(ctx, combine_partials_kernel, blocks, 256 * COMB_SPLIT, 0,
                      segs.as<double>(), mc.tmulti_row.as<int32_t>(),
                      mc.tmulti_first.as<int32_t>(), mc.tmulti_count.as<int32_t>(), mc.tmulti, P,
                      Yc);
        }
        if (timer) {
            // Bytes this layout must move: per nonzero its i_E (int32) and
            // value, per fibre its i_F and pointer (int32), each other factor
            // once, and the compact Y_(n) rows written.
            const double bytes = (double)sp->nnz * 12.0 + (double)mc.nfib * 8.0 +
                                 (double)mc.nrows * P * 8.0 +
                                 (double)sp->shape[F] * R[F] * 8.0 +
                                 (double)sp->shape[E] * R[E] * 8.0;
            timer->end(bytes);
        }
        return;
    }
    FactorSet f{};
    int d = 0;
    for (int m = 0; m < nd; m++) {
        if (m == mode) continue;
        f.U[d] = Ut_dev[m];
        f.R[d] = (int)R[m];
        d++;
    }
    DevMem part(ctx, std::max<int64_t>(mc.nslots, 1) * P * sizeof(double));
    if (timer) timer->begin();
    const int PL = (P + 31) / 32;
    if (PL <= 1) launch_rows<1>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    else if (PL <= 2) launch_rows<2>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    else if (PL <= 4) launch_rows<4>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    else if (PL <= 8) launch_rows<8>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    else if (PL <= 16) launch_rows<16>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    else launch_rows<32>(ctx, mc, nd - 1, sp->nnz, f, P, Yc, part.as<double>());
    if (mc.nmulti > 0) {
        const unsigned blocks = (unsigned)std::min<int64_t>(mc.nmulti, 65535);
        DT_LAUNCH(ctx, combine_partials_kernel, blocks, 256 * COMB_SPLIT, 0, part.as<double>(),
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
    SummaryScope sc(ctx, "Function::ttmc_mTR()", 2.0 * mc.nrows * P * Rn,
                    8.0 * mc.nrows * (P + Rn));
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
    DT_LAUNCH(ctx, sum_blocks_kernel, std::max(1u, std::min<unsigned>(ceil_div(n, 64), 65535)),
              256, 0, part.as<double>(), nblk, n, L);
}

void sp_mtl(dt_ctx *ctx, const dt_sptensor *sp, const double *Yc, int mode, int P,
            const double *L, int Rn, double *out) {
    const ModeCopy &mc = sp->modes[mode];
    SummaryScope sc(ctx, "Function::ttmc_mTL()", 2.0 * mc.nrows * P * Rn,
                    8.0 * mc.nrows * (P + Rn));
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
        sp->coo.idx.release();
        sp->coo.val.release();
        sp->dense_rows.clear();
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
            // The COO copy read by the general TTMc to a dense output.
            sp->coo.idx.alloc(ctx, (size_t)ndim * nnz * sizeof(int32_t));
            for (int m = 0; m < ndim; m++)
                DT_CUDA(cudaMemcpyAsync(sp->coo.idx.as<int32_t>() + (int64_t)m * nnz,
                                        idx32[m].get(), nnz * sizeof(int32_t),
                                        cudaMemcpyDeviceToDevice, ctx->stream));
            sp->coo.val.alloc(ctx, nnz * sizeof(double));
            DT_CUDA(cudaMemcpyAsync(sp->coo.val.get(), v.ptr(), nnz * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
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
        SummaryScope sc(ctx, "Algorithm::SpTucker::Sp_HOOI_ALS()");
        DT_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
        for (int it = 0; it < max_sweeps; it++) {
            for (int n = 0; n < nd; n++) {
                const int P = (int)kron_len(R, nd, n);
                sp_ttmc_compact(ctx, sp, ptrs, R, n, Yc.as<double>(), &timer);
                sp_mtr(ctx, sp, Yc.as<double>(), n, P, ptrs[n], (int)R[n], L.as<double>());
                sp_mtl(ctx, sp, Yc.as<double>(), n, P, L.as<double>(), (int)R[n],
                       const_cast<double *>(ptrs[n]));
                SummaryScope so(ctx, "Operator::orth2()", 2.0 * R[n] * R[n] * sp->shape[n],
                                8.0 * R[n] * sp->shape[n]);
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
        if (!std::isfinite(hg2)) fail(DT_ERR_NUMERIC, "sparse HOOI produced a non-finite core");
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
