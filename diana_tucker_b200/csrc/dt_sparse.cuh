// Device layout of a sparse tensor (dt_sptensor): one copy of the nonzeros
// per mode, in the row layout (any order) or the fibre layout (3-way), plus
// the COO copy the general TTMc to a dense output reads.
#pragma once

#include <map>
#include <memory>
#include <vector>

#include "dt_core.cuh"

namespace dt {

constexpr int MAXD = 8;

struct ModeCopy {
    int64_t nrows = 0;  // non-empty rows
    DevMem rows;        // int32 [nrows]: row id of compact row k
    // Row-kernel layout (orders other than 3): nonzeros sorted by this mode's
    // index, cut into chunks of at most CHUNK nonzeros.
    DevMem other;       // int32 [ndim-1][nnz]: the other modes' indices, in mode order
    DevMem val;         // double [nnz]
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
    // Fibre layout (3-way): nonzeros ordered by (row, fibre); a row's fibres,
    // cut into sub-fibres of at most FIB_CHUNK nonzeros, come longest first
    // and are padded with empty fibres to a multiple of 4 (a group).
    int fmode = -1;       // fibre mode F; the element mode E is the remaining one
    int64_t nfib = 0;     // fibre slots (4 per group)
    DevMem e_idx;         // int32 [nnz]: i_E of each nonzero, in fibre order
    DevMem e_val;         // double [nnz]
    DevMem fib_idx;       // int32 [nfib]: i_F of each fibre slot (0 when empty)
    DevMem fib_ptr;       // int32 [nfib+1]: its nonzeros
    DevMem grp_row;       // int32 [nfib/4]: compact row of each group
    DevMem grp_aux;       // int32 [nfib/4]: longest fibre | FB_ROW_END (last group of its row)
    // Batches: int2 {first group, first nonzero} (+ an end entry); a batch is
    // at most FB_GRP groups and FB_NZ nonzeros.  Tasks: int4 {first batch, end
    // batch, partial slot or -1, 0}: packs of whole consecutive rows, or pieces
    // of one long row, largest first.
    int64_t nbatch = 0;
    DevMem batches;
    int64_t ntasks = 0;
    DevMem tasks;
    int64_t tslots = 0;
    int64_t tmulti = 0;   // rows cut into several pieces
    // Their partial rows are summed in two levels: segments of at most
    // COMB_SEG consecutive pieces (tseg_first / tseg_count: piece slots), then
    // each row's segments (tmulti_first / tmulti_count: segment indices).
    DevMem tmulti_row, tmulti_first, tmulti_count;
    int64_t nseg = 0;
    DevMem tseg_first, tseg_count;
};

struct FactorSet {
    const double *U[MAXD];  // transposed factors: row i of mode m at U[m] + i*R[m]
    int R[MAXD];
};

// The nonzeros in input order: int32 indices (mode-major, ndim x nnz) and
// FP64 values.
struct SpCoo {
    DevMem idx;  // int32 [ndim][nnz]
    DevMem val;  // double [nnz]
};

}  // namespace dt

struct dt_sptensor {
    dt_ctx *ctx = nullptr;
    int ndim = 0;
    int64_t nnz = 0;
    int64_t shape[dt::MAXD] = {};
    double fnorm = 0.0;
    std::vector<dt::ModeCopy> modes;
    dt::SpCoo coo;
    // Row groupings of the nonzeros for dt_sp_ttmc_dense_f64, one per set of
    // kept (not contracted) modes (bit mask), built on first use.
    std::map<unsigned, std::shared_ptr<void>> dense_rows;
};

