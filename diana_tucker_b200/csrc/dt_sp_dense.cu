// The general sparse TTMc to a dense output, Function::ttmc(SpTensor, M, idx,
// distribution, to_permu) (template/function/sp_tensor.tpp:16-192, with the
// recursion of add_outer_product, :419-450), and Function::mettmc (:194-211),
// at world size 1.
//
//   Y = A x_{m in idx} M_m,   M_m J_m x I_m col-major,
//
// a dense column-major tensor whose contracted modes have extent J_m and whose
// other ("kept") modes keep I_m.  Every nonzero adds v (x)_{m in idx} M_m(:, i_m)
// to the block of Y at its kept coordinates.  The reference accumulates into a
// per-rank buffer (and a ring of them across ranks); here the nonzeros are
// grouped by their kept coordinates once per set of kept modes (a radix sort
// of the kept-mode key, cached on the tensor) and every group ("row") is
// summed by one warp in a fixed order:
//
//  * a row of more than CH nonzeros is cut into pieces; each piece writes a
//    partial block, and a second kernel adds a row's pieces in order and
//    writes the block (no floating-point atomics, deterministic output);
//  * lane l of the warp owns the Kronecker entries p = l + 32 q (q < PL) of a
//    tile of 32 PL entries, the lowest contracted mode fastest; each nonzero's
//    value and contracted indices are broadcast by shuffles and every lane
//    multiplies the factor entries of its p's;
//  * rows (kept coordinates) without nonzeros stay zero.
//
// The reference's to_permu only chooses its internal buffer layout (contracted
// modes first, permuted back at the end, :170-182); the result is the same.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "dt_kernels.cuh"
#include "dt_sparse.cuh"

namespace dt {
namespace {

constexpr int DN_CH = 1024;  // nonzeros per piece of a row
constexpr int DN_PL = 8;     // Kronecker entries per lane in one tile
constexpr int DN_TILE = 32 * DN_PL;

struct DenseRows {
    int64_t nrows = 0, ntasks = 0, nslots = 0, nmulti = 0;
    DevMem perm;   // int32 [nnz]: nonzero ids grouped by kept coordinates
    DevMem tasks;  // int4 [ntasks]: {first position, end position, slot or -1, -}
    DevMem multi;  // int4 [nmulti]: {first position of the row, first slot, pieces, -}
};

struct DenseArgs {
    const int32_t *idx;  // COO indices, mode-major
    const double *val;
    int64_t nnz;
    const int32_t *perm;
    int nc;                        // contracted modes
    int cmode[MAXD];               // their mode numbers, ascending
    const double *M[MAXD];         // their factors (J x I col-major)
    int64_t J[MAXD];
    int64_t cstride[MAXD];         // their output strides
    int nk;                        // kept modes
    int kmode[MAXD];
    int64_t kstride[MAXD];         // their output strides
    int64_t P;                     // prod_{contracted} J
};

__global__ void kept_key_kernel(const int32_t *__restrict__ idx, int64_t nnz, int nk,
                                const int *__restrict__ kmode_dev, const uint64_t *__restrict__ kst,
                                uint64_t *__restrict__ key, int32_t *__restrict__ ids) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = 0;
        for (int d = 0; d < nk; d++) k += (uint64_t)idx[(int64_t)kmode_dev[d] * nnz + e] * kst[d];
        key[e] = k;
        ids[e] = (int32_t)e;
    }
}

// Output offset of a row (kept coordinates of the nonzero id e).
__device__ __forceinline__ int64_t row_base(const DenseArgs &a, int32_t e) {
    int64_t b = 0;
    for (int d = 0; d < a.nk; d++) b += (int64_t)a.idx[(int64_t)a.kmode[d] * a.nnz + e] * a.kstride[d];
    return b;
}

// Output offset of Kronecker entry p (lowest contracted mode fastest).
__device__ __forceinline__ int64_t kron_offset(const DenseArgs &a, int64_t p) {
    int64_t o = 0;
    for (int d = 0; d < a.nc; d++) {
        o += (p % a.J[d]) * a.cstride[d];
        p /= a.J[d];
    }
    return o;
}

constexpr int DN_WARPS = 4;  // warps per CTA of the TTMc kernel

__global__ void __launch_bounds__(32 * DN_WARPS) dense_ttmc_kernel(DenseArgs a, const int4 *__restrict__ tasks,
                                                         int64_t ntasks, int64_t ntiles,
                                                         double *__restrict__ Y,
                                                         double *__restrict__ part) {
    // Per warp: the contracted digits of the lane's entries, [q][d][lane]
    // (32 KB per CTA).
    __shared__ int32_t dig[DN_WARPS][DN_PL][MAXD][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int64_t cur_tile = -1;
    for (int64_t wi = warp0; wi < ntasks * ntiles; wi += nwarps) {
        const int64_t task = wi / ntiles, tile = wi % ntiles;
        const int64_t p0 = tile * DN_TILE;
        if (tile != cur_tile) {
            cur_tile = tile;
            __syncwarp();  // every lane is done reading the previous tile's digits
#pragma unroll
            for (int q = 0; q < DN_PL; q++) {
                int64_t p = p0 + lane + 32 * q;
                for (int d = 0; d < a.nc; d++) {
                    dig[w][q][d][lane] = (int32_t)(p % a.J[d]);
                    p /= a.J[d];
                }
            }
            __syncwarp();
        }
        const int4 tk = tasks[task];
        double acc[DN_PL];
#pragma unroll
        for (int q = 0; q < DN_PL; q++) acc[q] = 0.0;
        for (int beg = tk.x; beg < tk.y; beg += 32) {
            const int pos = beg + lane;
            const bool ok = pos < tk.y;
            const int32_t e = ok ? a.perm[pos] : 0;
            const double myv = ok ? a.val[e] : 0.0;
            int32_t myi[MAXD];
#pragma unroll
            for (int d = 0; d < MAXD; d++)
                myi[d] = (d < a.nc && ok) ? a.idx[(int64_t)a.cmode[d] * a.nnz + e] : 0;
            const int cnt = min(32, tk.y - beg);
            for (int j = 0; j < cnt; j++) {
                const double v = __shfl_sync(0xffffffffu, myv, j);
                int64_t col[MAXD];
#pragma unroll
                for (int d = 0; d < MAXD; d++)
                    col[d] = (int64_t)__shfl_sync(0xffffffffu, myi[d], j) * a.J[d < a.nc ? d : 0];
#pragma unroll
                for (int q = 0; q < DN_PL; q++) {
                    double prod = v;
                    for (int d = 0; d < a.nc; d++) prod *= a.M[d][dig[w][q][d][lane] + col[d]];
                    acc[q] += prod;
                }
            }
        }
        if (tk.z < 0) {
            const int64_t base = row_base(a, a.perm[tk.x]);
#pragma unroll
            for (int q = 0; q < DN_PL; q++) {
                const int64_t p = p0 + lane + 32 * q;
                if (p < a.P) Y[base + kron_offset(a, p)] = acc[q];
            }
        } else {
            double *dst = part + (int64_t)tk.z * a.P;
#pragma unroll
            for (int q = 0; q < DN_PL; q++) {
                const int64_t p = p0 + lane + 32 * q;
                if (p < a.P) dst[p] = acc[q];
            }
        }
    }
}

// Rows cut into pieces: entry p of row r is the sum of its pieces' partials,
// in piece order.  grid.x: rows, grid.y x block: entries.
__global__ void __launch_bounds__(256) dense_combine_kernel(DenseArgs a,
                                                            const int4 *__restrict__ multi,
                                                            const double *__restrict__ part,
                                                            double *__restrict__ Y) {
    const int4 m = multi[blockIdx.x];
    const int64_t base = row_base(a, a.perm[m.x]);
    for (int64_t p = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; p < a.P;
         p += (int64_t)gridDim.y * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < m.z; k++) s += part[(int64_t)(m.y + k) * a.P + p];
        Y[base + kron_offset(a, p)] = s;
    }
}

// Groups the nonzeros by their coordinates in the kept modes (bit mask) and
// cuts the groups into pieces of at most DN_CH nonzeros.
std::shared_ptr<DenseRows> build_dense_rows(dt_ctx *ctx, const dt_sptensor *sp, unsigned kept) {
    auto dr = std::make_shared<DenseRows>();
    const int64_t nnz = sp->nnz;
    std::vector<int> km;
    std::vector<uint64_t> kst;
    uint64_t s = 1;
    int bits = 0;
    for (int m = 0; m < sp->ndim; m++) {
        if (!(kept >> m & 1u)) continue;
        km.push_back(m);
        kst.push_back(s);
        s *= (uint64_t)sp->shape[m];
    }
    while (bits < 64 && (uint64_t(1) << bits) < s) bits++;
    DevMem key(ctx, nnz * sizeof(uint64_t)), key2(ctx, nnz * sizeof(uint64_t));
    DevMem ids(ctx, nnz * sizeof(int32_t));
    dr->perm.alloc(ctx, nnz * sizeof(int32_t));
    DevMem dkm(ctx, std::max<size_t>(1, km.size()) * sizeof(int));
    DevMem dkst(ctx, std::max<size_t>(1, kst.size()) * sizeof(uint64_t));
    if (!km.empty()) {
        DT_CUDA(cudaMemcpyAsync(dkm.get(), km.data(), km.size() * sizeof(int),
                                cudaMemcpyHostToDevice, ctx->stream));
        DT_CUDA(cudaMemcpyAsync(dkst.get(), kst.data(), kst.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice, ctx->stream));
    }
    const unsigned blocks = std::max(1u, std::min<unsigned>(ceil_div(nnz, 256), 8u * ctx->num_sms));
    DT_LAUNCH(ctx, kept_key_kernel, blocks, 256, 0, sp->coo.idx.as<int32_t>(), nnz, (int)km.size(),
              dkm.as<int>(), dkst.as<uint64_t>(), key.as<uint64_t>(), ids.as<int32_t>());
    // Stable radix sort of (key, id): a group keeps its nonzeros in input order.
    size_t tmp_bytes = 0;
    if (bits > 0) {
        DT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.as<uint64_t>(),
                                                key2.as<uint64_t>(), ids.as<int32_t>(),
                                                dr->perm.as<int32_t>(), (int)nnz, 0, bits,
                                                ctx->stream));
        DevMem tmp(ctx, std::max<size_t>(tmp_bytes, 1));
        DT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, key.as<uint64_t>(),
                                                key2.as<uint64_t>(), ids.as<int32_t>(),
                                                dr->perm.as<int32_t>(), (int)nnz, 0, bits,
                                                ctx->stream));
    } else {
        // Nothing kept: one group, input order.
        DT_CUDA(cudaMemcpyAsync(key2.get(), key.get(), nnz * sizeof(uint64_t),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        DT_CUDA(cudaMemcpyAsync(dr->perm.get(), ids.get(), nnz * sizeof(int32_t),
                                cudaMemcpyDeviceToDevice, ctx->stream));
    }
    // Group lengths (run-length encoding of the sorted keys).
    DevMem uniq(ctx, nnz * sizeof(uint64_t)), counts(ctx, nnz * sizeof(int32_t));
    DevMem nruns(ctx, sizeof(int32_t));
    tmp_bytes = 0;
    DT_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tmp_bytes, key2.as<uint64_t>(),
                                               uniq.as<uint64_t>(), counts.as<int32_t>(),
                                               nruns.as<int32_t>(), (int)nnz, ctx->stream));
    {
        DevMem tmp(ctx, std::max<size_t>(tmp_bytes, 1));
        DT_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.get(), tmp_bytes, key2.as<uint64_t>(),
                                                   uniq.as<uint64_t>(), counts.as<int32_t>(),
                                                   nruns.as<int32_t>(), (int)nnz, ctx->stream));
    }
    int32_t hn = 0;
    DT_CUDA(cudaMemcpyAsync(&hn, nruns.get(), sizeof(int32_t), cudaMemcpyDeviceToHost,
                            ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> cnt(hn);
    DT_CUDA(cudaMemcpyAsync(cnt.data(), counts.get(), (size_t)hn * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, ctx->stream));
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    // Pieces, longest rows first in the task list (their pieces are spread
    // over many warps early), partial slots for rows of more than one piece.
    std::vector<int4> tasks, multi;
    std::vector<int64_t> start(hn + 1, 0);
    for (int32_t r = 0; r < hn; r++) start[r + 1] = start[r] + cnt[r];
    std::vector<int32_t> order(hn);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return cnt[x] > cnt[y]; });
    int32_t slot = 0;
    for (int32_t r : order) {
        const int32_t b = (int32_t)start[r], e = (int32_t)start[r + 1];
        const int32_t pieces = (cnt[r] + DN_CH - 1) / DN_CH;
        if (pieces == 1) {
            tasks.push_back(make_int4(b, e, -1, 0));
        } else {
            multi.push_back(make_int4(b, slot, pieces, 0));
            for (int32_t k = 0; k < pieces; k++)
                tasks.push_back(make_int4(b + k * DN_CH, std::min(e, b + (k + 1) * DN_CH),
                                          slot + k, 0));
            slot += pieces;
        }
    }
    dr->nrows = hn;
    dr->ntasks = (int64_t)tasks.size();
    dr->nslots = slot;
    dr->nmulti = (int64_t)multi.size();
    dr->tasks.alloc(ctx, std::max<size_t>(1, tasks.size()) * sizeof(int4));
    DT_CUDA(cudaMemcpyAsync(dr->tasks.get(), tasks.data(), tasks.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, ctx->stream));
    if (!multi.empty()) {
        dr->multi.alloc(ctx, multi.size() * sizeof(int4));
        DT_CUDA(cudaMemcpyAsync(dr->multi.get(), multi.data(), multi.size() * sizeof(int4),
                                cudaMemcpyHostToDevice, ctx->stream));
    }
    DT_CUDA(cudaStreamSynchronize(ctx->stream));
    return dr;
}

// Y (device, prod of the output extents) = A x_{m in contracted} M_m.
// M[m] (device, J[m] x I_m col-major) for every contracted mode.
void sp_ttmc_dense(dt_ctx *ctx, dt_sptensor *sp, const double *const *M, const int64_t *J,
                   unsigned contracted, double *Y) {
    const int N = sp->ndim;
    unsigned kept = 0;
    for (int m = 0; m < N; m++)
        if (!(contracted >> m & 1u)) kept |= 1u << m;
    auto it = sp->dense_rows.find(kept);
    if (it == sp->dense_rows.end())
        it = sp->dense_rows.emplace(kept, build_dense_rows(ctx, sp, kept)).first;
    const DenseRows &dr = *std::static_pointer_cast<DenseRows>(it->second);
    DenseArgs a{};
    a.idx = sp->coo.idx.as<int32_t>();
    a.val = sp->coo.val.as<double>();
    a.nnz = sp->nnz;
    a.perm = dr.perm.as<int32_t>();
    int64_t stride = 1, total = 1;
    a.P = 1;
    for (int m = 0; m < N; m++) {
        const bool c = contracted >> m & 1u;
        const int64_t ext = c ? J[m] : sp->shape[m];
        if (c) {
            a.cmode[a.nc] = m;
            a.M[a.nc] = M[m];
            a.J[a.nc] = J[m];
            a.cstride[a.nc] = stride;
            a.nc++;
            a.P *= J[m];
        } else {
            a.kmode[a.nk] = m;
            a.kstride[a.nk] = stride;
            a.nk++;
        }
        stride *= ext;
        total *= ext;
    }
    DT_CUDA(cudaMemsetAsync(Y, 0, total * sizeof(double), ctx->stream));
    const int64_t ntiles = (a.P + DN_TILE - 1) / DN_TILE;
    DevMem part(ctx, std::max<int64_t>(1, dr.nslots) * a.P * sizeof(double));
    const int64_t work = dr.ntasks * ntiles;
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((work + DN_WARPS - 1) / DN_WARPS, 32LL * ctx->num_sms));
    DT_LAUNCH(ctx, dense_ttmc_kernel, blocks, 32 * DN_WARPS, 0, a, dr.tasks.as<int4>(), dr.ntasks,
              ntiles, Y, part.as<double>());
    if (dr.nmulti > 0) {
        const unsigned gy = (unsigned)std::min<int64_t>((a.P + 255) / 256, 64);
        DT_LAUNCH(ctx, dense_combine_kernel, dim3((unsigned)dr.nmulti, gy), 256, 0, a,
                  dr.multi.as<int4>(), part.as<double>(), Y);
    }
}

void check_dense_args(const dt_sptensor *sp, const double *const *M, const int64_t *J,
                      const int *idx, int nidx, unsigned *mask, const char *who) {
    DT_CHECK_ARG(nidx >= 0 && nidx <= sp->ndim && (nidx == 0 || (idx && M && J)),
                 "%s: bad mode list", who);
    unsigned c = 0;
    for (int k = 0; k < nidx; k++) {
        const int m = idx[k];
        DT_CHECK_ARG(m >= 0 && m < sp->ndim, "%s: mode %d out of range", who, m);
        DT_CHECK_ARG(!(c >> m & 1u), "%s: mode %d listed twice", who, m);
        DT_CHECK_ARG(M[m] && J[m] >= 1 && J[m] < (int64_t(1) << 31),
                     "%s: factor of mode %d missing or J = %lld out of range", who, m,
                     (long long)J[m]);
        c |= 1u << m;
    }
    int64_t total = 1;
    for (int m = 0; m < sp->ndim; m++) {
        const int64_t ext = (c >> m & 1u) ? J[m] : sp->shape[m];
        DT_CHECK_ARG(ext <= (int64_t(1) << 62) / total, "%s: the output is too large", who);
        total *= ext;
    }
    *mask = c;
}

}  // namespace

void sp_release_dense_rows(dt_sptensor *sp) { sp->dense_rows.clear(); }

}  // namespace dt

using namespace dt;

namespace {

void check_sp_ctx(const dt_ctx *ctx, const dt_sptensor *sp) {
    check_ctx(ctx);
    DT_CHECK_ARG(sp, "null dt_sptensor");
    DT_CHECK_ARG(sp->ctx == ctx, sp->ctx ? "dt_sptensor belongs to another dt_ctx"
                                         : "dt_sptensor's dt_ctx was destroyed");
}

int64_t out_size(const dt_sptensor *sp, const int64_t *J, unsigned c) {
    int64_t t = 1;
    for (int m = 0; m < sp->ndim; m++) t *= (c >> m & 1u) ? J[m] : sp->shape[m];
    return t;
}

struct FactorViews {
    std::vector<DevView> views;
    const double *ptrs[MAXD] = {};
};

void view_factors(dt_ctx *ctx, const dt_sptensor *sp, const double *const *M, const int64_t *J,
                  unsigned c, FactorViews &fv) {
    fv.views.reserve(sp->ndim);
    for (int m = 0; m < sp->ndim; m++) {
        if (!(c >> m & 1u)) continue;
        fv.views.emplace_back(ctx, M[m], (size_t)J[m] * sp->shape[m] * sizeof(double), true, false);
        fv.ptrs[m] = fv.views.back().as<double>();
    }
}

}  // namespace

extern "C" {

int dt_sp_ttmc_dense_f64(dt_ctx *ctx, const dt_sptensor *sp, const double *const *M,
                         const int64_t *J, const int *idx, int nidx, double *Y) {
    return guard([&] {
        check_sp_ctx(ctx, sp);
        DT_CHECK_ARG(Y, "dt_sp_ttmc_dense_f64: null output");
        unsigned c = 0;
        check_dense_args(sp, M, J, idx, nidx, &c, "dt_sp_ttmc_dense_f64");
        DT_CUDA(cudaSetDevice(ctx->device));
        SummaryScope sc(ctx, "Function::ttmc()");
        FactorViews fv;
        view_factors(ctx, sp, M, J, c, fv);
        DevView y(ctx, Y, out_size(sp, J, c) * sizeof(double), false, true);
        sp_ttmc_dense(ctx, const_cast<dt_sptensor *>(sp), fv.ptrs, J, c, y.as<double>());
        y.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int dt_sp_mettmc_f64(dt_ctx *ctx, const dt_sptensor *sp, const double *const *M,
                     const int64_t *J, const int *idx, int nidx, int level, double *Y) {
    return guard([&] {
        check_sp_ctx(ctx, sp);
        DT_CHECK_ARG(Y, "dt_sp_mettmc_f64: null output");
        unsigned c = 0;
        check_dense_args(sp, M, J, idx, nidx, &c, "dt_sp_mettmc_f64");
        DT_CHECK_ARG(level >= 0 && level <= nidx, "dt_sp_mettmc_f64: level %d not in [0, %d]",
                     level, nidx);
        DT_CUDA(cudaSetDevice(ctx->device));
        SummaryScope sc(ctx, "Function::mettmc()");
        // The modes ordered by I_m / J_m (integer quotient, ascending; ties
        // keep the caller's order): the first `level` are contracted densely
        // after the sparse TTMc of the others (sp_tensor.tpp:198-208).
        std::vector<int> ord(idx, idx + nidx);
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
            return sp->shape[x] / J[x] < sp->shape[y] / J[y];
        });
        unsigned csparse = 0;
        for (int k = level; k < nidx; k++) csparse |= 1u << ord[k];
        FactorViews fv;
        view_factors(ctx, sp, M, J, c, fv);
        DevView y(ctx, Y, out_size(sp, J, c) * sizeof(double), false, true);
        int64_t shape[MAXD];
        for (int m = 0; m < sp->ndim; m++) shape[m] = (csparse >> m & 1u) ? J[m] : sp->shape[m];
        DevMem cur(ctx, out_size(sp, J, csparse) * sizeof(double));
        sp_ttmc_dense(ctx, const_cast<dt_sptensor *>(sp), fv.ptrs, J, csparse, cur.as<double>());
        for (int k = 0; k < level; k++) {
            const int m = ord[k];
            int64_t L = 1, B = 1;
            for (int q = 0; q < m; q++) L *= shape[q];
            for (int q = m + 1; q < sp->ndim; q++) B *= shape[q];
            double *dst;
            DevMem nxt;
            if (k + 1 == level) {
                dst = y.as<double>();
            } else {
                nxt.alloc(ctx, L * J[m] * B * sizeof(double));
                dst = nxt.as<double>();
            }
            // Function::ttm(Y, M_m, m): Y x_m M_m with M_m J_m x I_m col-major.
            ttm_f64<double>(ctx, cur.as<double>(), L, shape[m], B, fv.ptrs[m], 1, J[m], J[m], dst);
            shape[m] = J[m];
            if (k + 1 < level) cur = std::move(nxt);
        }
        if (level == 0)
            DT_CUDA(cudaMemcpyAsync(y.ptr(), cur.get(), out_size(sp, J, c) * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
        y.finish();
        DT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"
