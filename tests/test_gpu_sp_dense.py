"""The general sparse TTMc to a dense output (Function::ttmc(SpTensor, ...),
sp_tensor.tpp:16-192) and Function::mettmc (sp_tensor.tpp:194-211) on the GPU,
against the C restatement of the reference's add_outer_product recursion
(oracle/sparse_oracle.c, itself pinned to the reference's Function::ttm on
the densified tensor by tests/test_oracle.py).

Tolerance: 1e-12 relative to the largest entry (FP64 in both; the sums run
in different orders)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / max(1e-300, np.max(np.abs(b))))


def _tensor(shape, nnz, seed, dup=True):
    rng = np.random.default_rng(seed)
    keys = rng.choice(int(np.prod(shape)), size=nnz, replace=False)
    idx = [np.asarray(i, dtype=np.int64) for i in np.unravel_index(keys, shape, order="F")]
    vals = rng.lognormal(0, 1, nnz)
    if dup:
        rep = rng.choice(nnz, size=nnz // 4, replace=False)
        idx = [np.concatenate([i, i[rep]]) for i in idx]
        vals = np.concatenate([vals, rng.lognormal(0, 1, rep.size)])
    M = [np.asfortranarray(rng.standard_normal((2 + (m % 4) * 3, s)))
         for m, s in enumerate(shape)]
    return idx, vals, list(shape), M


CASES = [((30, 20, 10), []), ((30, 20, 10), [1]), ((30, 20, 10), [0, 2]),
         ((30, 20, 10), [2, 0, 1]), ((12, 9, 8, 7), [3, 0]), ((12, 9, 8, 7), [0, 1, 2, 3]),
         ((6, 5, 4, 3, 4), [4, 2, 1])]


@pytest.mark.parametrize("shape,modes", CASES)
def test_ttmc_dense_vs_oracle(ctx, oracle_sparse, shape, modes):
    idx, vals, shape, M = _tensor(shape, 900 if len(shape) < 5 else 400, 3)
    sp = ctx.sptensor(idx, vals, shape)
    try:
        Y = sp.ttmc_dense(M, modes)
        Y2 = sp.ttmc_dense(M, modes)  # the cached grouping, and determinism
    finally:
        sp.close()
    Yo = oracle_sparse.ttmc_dense(idx, vals, shape, M, modes)
    assert Y.shape == Yo.shape
    assert _rel(Y, Yo) <= 1e-12
    assert np.array_equal(Y, Y2)


@pytest.mark.parametrize("shape,modes", [((30, 20, 10), [0, 1, 2]), ((12, 9, 8, 7), [3, 1, 0])])
def test_mettmc_every_level_vs_oracle(ctx, oracle_sparse, shape, modes):
    idx, vals, shape, M = _tensor(shape, 900, 5)
    Yo = oracle_sparse.ttmc_dense(idx, vals, shape, M, modes)
    sp = ctx.sptensor(idx, vals, shape)
    try:
        for level in range(len(modes) + 1):
            assert _rel(sp.mettmc(M, modes, level), Yo) <= 1e-12, level
    finally:
        sp.close()


def test_ttmc_dense_long_rows_and_wide_blocks(ctx, oracle_sparse):
    """Zipf rows of thousands of nonzeros (cut into pieces, combined in order)
    and a Kronecker block wider than one tile (P = 24 x 20 = 480)."""
    from diana_tucker_b200 import datasets
    idx, vals, shape = datasets.sparse_zipf((400, 300, 50), 60_000, alpha=1.3, seed=4)
    rng = np.random.default_rng(6)
    M = [np.asfortranarray(rng.standard_normal((j, s))) for j, s in zip((24, 20, 9), shape)]
    sp = ctx.sptensor(idx, vals, shape)
    try:
        for modes in ([0, 1], [1, 2], [0, 1, 2]):
            Y = sp.ttmc_dense(M, modes)
            assert _rel(Y, oracle_sparse.ttmc_dense(idx, vals, shape, M, modes)) <= 1e-12, modes
    finally:
        sp.close()


def test_ttmc_dense_agrees_with_ttmc_rows(ctx):
    """Contracting every mode but n with the transposed factors is the TTMc of
    the HOOI path (dt_sp_ttmc_rows, Y_(n) row-major), laid out column-major."""
    from diana_tucker_b200 import datasets
    idx, vals, shape = datasets.sparse_zipf((5000, 3000, 800), 200_000, seed=9)
    R = (8, 6, 5)
    Ut = datasets.random_orthonormal_transposed(shape, R, 3)
    sp = ctx.sptensor(idx, vals, shape)
    try:
        for n in range(3):
            others = [m for m in range(3) if m != n]
            Y = sp.ttmc_dense([u.T for u in Ut], others)  # M_m = U_m^T, R_m x I_m
            rows = sp.ttmc_rows(Ut, R, n)  # I_n x P, lower other mode fastest
            Yn = np.moveaxis(Y, n, 0).reshape(shape[n], -1, order="F")
            assert _rel(Yn, rows) <= 1e-12, n
    finally:
        sp.close()


def test_ttmc_dense_rejects_bad_modes(ctx):
    from diana_tucker_b200 import DTError
    idx, vals, shape, M = _tensor((6, 5, 4), 30, 1, dup=False)
    sp = ctx.sptensor(idx, vals, shape)
    try:
        with pytest.raises(DTError):
            sp.ttmc_dense(M, [0, 0])
        with pytest.raises(DTError):
            sp.mettmc(M, [0, 1], 3)
    finally:
        sp.close()
