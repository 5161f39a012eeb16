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

// mTL: out[:, rows[k]] = (Yc[k, :] L)^T, L is P x Rn col-major (in smem).
// One warp per compact row; empty rows of out are zeroed beforehand.
__global__ void __launch_bounds__(256) mtl_kernel(const double *__restrict__ Yc,
                                                  const int32_t *__restrict__ rows,
                                                  int64_t nrows, int P, const double *__restrict__ L,
                                                  int Rn, double *__restrict__ out) {
    extern __shared__ double Ls[];
    for (int e = threadIdx.x; e < P * Rn; e += blockDim.x) Ls[e] = L[e];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = warp0; k < nrows; k += nwarps) {
        const double *y = Yc + k * P;
        double mine = 0.0;  // lane r < Rn ends up holding output r
        for (int r = 0; r < Rn; r++) {
            double s = 0.0;
            for (int p = lane; p < P; p += 32) s = fma(y[p], Ls[p + (int64_t)P * r], s);
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == (r & 31)) mine = s;
            if ((r & 31) == 31 || r == Rn - 1) {
                const int base = r & ~31;
                if (lane <= (r & 31)) out[(int64_t)rows[k] * Rn + base + lane] = mine;
            }
        }
    }
}

// mTR partials: part[blk][p + P*r] = sum over this block's compact rows of
// Yc[k, p] * U_n(rows[k], r).  Thread t owns entries p = t, t + blockDim, ...
// and keeps the R_n (<= 32) sums of its entry in registers.
__global__ void __launch_bounds__(256) mtr_partial_kernel(const double *__restrict__ Yc,
                                                          const int32_t *__restrict__ rows,
                                                          int64_t nrows, int P,
                                                          const double *__restrict__ Un, int Rn,
                                                          int64_t rows_per_block,
                                                          double *__restrict__ part) {
    extern __shared__ double us[];  // staged U_n rows: [batch][Rn]
    constexpr int BATCH = 32;
    const int64_t k0 = blockIdx.x * rows_per_block;
    const int64_t k1 = min(nrows, k0 + rows_per_block);
    for (int p0 = 0; p0 < P; p0 += blockDim.x) {
        const int p = p0 + threadIdx.x;
        double acc[32];
#pragma unroll
        for (int r = 0; r < 32; r++) acc[r] = 0.0;
        for (int64_t kb = k0; kb < k1; kb += BATCH) {
            const int nb = (int)(k1 - kb < BATCH ? k1 - kb : BATCH);
            __syncthreads();
            for (int e = threadIdx.x; e < nb * Rn; e += blockDim.x) {
                const int b = e / Rn, r = e % Rn;
                us[e] = Un[(int64_t)rows[kb + b] * Rn + r];
            }
            __syncthreads();
            if (p < P) {
                for (int b = 0; b < nb; b++) {
                    const double yv = Yc[(kb + b) * P + p];
#pragma unroll
                    for (int r = 0; r < 32; r++)
                        if (r < Rn) acc[r] = fma(yv, us[b * Rn + r], acc[r]);
                }
            }
        }
        if (p < P) {
#pragma unroll
            for (int r = 0; r < 32; r++)
                if (r < Rn) part[(int64_t)blockIdx.x * P * Rn + p + (int64_t)P * r] = acc[r];
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
    DT_LAUNCH(ctx, mtr_partial_kernel, nblk, 256, 32 * Rn * sizeof(double), Yc,
              mc.rows.as<int32_t>(), mc.nrows, P, Un, Rn, rpb, part.as<double>());
    const int64_t n = (int64_t)P * Rn;
    DT_LAUNCH(ctx, sum_blocks_kernel, std::max(1u, ceil_div(n, 256)), 256, 0,
              part.as<double>(), nblk, n, L);
}

void sp_mtl(dt_ctx *ctx, const dt_sptensor *sp, const double *Yc, int mode, int P,
            const double *L, int Rn, double *out) {
    const ModeCopy &mc = sp->modes[mode];
    DT_CUDA(cudaMemsetAsync(out, 0, sp->shape[mode] * Rn * sizeof(double), ctx->stream));
    const size_t smem = (size_t)P * Rn * sizeof(double);
    DT_CHECK_ARG(smem <= 200 * 1024, "sparse ttmc_mTL: L (%d x %d) too large", P, Rn);
    DT_CUDA(cudaFuncSetAttribute(mtl_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    const unsigned blocks =
        std::max(1u, std::min<unsigned>(ceil_div(mc.nrows, 8), 8u * (unsigned)ctx->num_sms));
    DT_LAUNCH(ctx, mtl_kernel, blocks, 256, smem, Yc, mc.rows.as<int32_t>(), mc.nrows, P, L,
              Rn, out);
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
        *out = sp;
    });
}

int dt_sptensor_destroy(dt_sptensor *sp) {
    return guard([&] {
        if (!sp) return;
        cudaSetDevice(sp->ctx->device);
        cudaStreamSynchronize(sp->ctx->stream);
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
