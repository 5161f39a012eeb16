"""Sparse TTMc and sparse HOOI on the GPU vs the C restatement (oracle).

Tolerance: 1e-12 relative (FP64; only the summation order differs)."""
import numpy as np
import pytest

from oracle import dense

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b)))


@pytest.fixture(scope="module")
def zipf_small():
    from diana_tucker_b200 import datasets
    # Zipf heads give rows far longer than one 512-nonzero chunk.
    return datasets.sparse_zipf((3000, 500, 200), 40000, alpha=1.1, seed=12)


def _factors(shape, R, seed):
    from diana_tucker_b200 import datasets
    return datasets.random_orthonormal_transposed(shape, R, seed)


@pytest.mark.parametrize("R", [(16, 16, 16), (8, 4, 2), (5, 3, 7), (8, 16, 16), (16, 8, 8),
                               (32, 32, 32), (10, 10, 10), (12, 12, 12), (4, 4, 4)])
def test_ttmc_rows_mtr_mtl(ctx, oracle_sparse, zipf_small, R):
    idx, vals, shape = zipf_small
    sp = ctx.sptensor(idx, vals, shape)
    Ut = _factors(shape, R, 1)
    assert abs(sp.fnorm() - np.linalg.norm(vals)) < 1e-12 * np.linalg.norm(vals)
    for mode in range(3):
        Y = sp.ttmc_rows(Ut, R, mode)
        Yo = oracle_sparse.ttmc_rows(idx, vals, shape, Ut, R, mode)
        assert _rel(Y, Yo) < 1e-12
        L = sp.ttmc_mTR(Ut, R, mode)
        Lo = oracle_sparse.ttmc_mTR(idx, vals, shape, Ut, R, mode)
        assert _rel(L, Lo) < 1e-12
        out = sp.ttmc_mTL(Ut, R, mode, Lo)
        outo = oracle_sparse.ttmc_mTL(idx, vals, shape, Ut, R, mode, Lo)
        assert _rel(out, outo) < 1e-12
    sp.close()


@pytest.mark.parametrize("R", [(4, 40, 24), (33, 2, 30)])
def test_ttmc_wide_ranks(ctx, oracle_sparse, zipf_small, R):
    """Other-mode ranks above 32 (P <= 1024) take the wide fibre kernel."""
    idx, vals, shape = zipf_small
    sp = ctx.sptensor(idx, vals, shape)
    Ut = _factors(shape, R, 7)
    for mode in range(3):
        P = int(np.prod([R[m] for m in range(3) if m != mode]))
        if P > 1024:
            continue
        Y = sp.ttmc_rows(Ut, R, mode)
        assert _rel(Y, oracle_sparse.ttmc_rows(idx, vals, shape, Ut, R, mode)) < 1e-12
    sp.close()


def test_sparse_four_way_generic_path(ctx, oracle_sparse):
    from diana_tucker_b200 import datasets
    idx, vals, shape = datasets.sparse_zipf((60, 40, 30, 20), 5000, alpha=1.1, seed=4)
    R = (3, 2, 4, 2)
    Ut = _factors(shape, R, 2)
    sp = ctx.sptensor(idx, vals, shape)
    for mode in range(4):
        assert _rel(sp.ttmc_rows(Ut, R, mode),
                    oracle_sparse.ttmc_rows(idx, vals, shape, Ut, R, mode)) < 1e-12
        assert _rel(sp.ttmc_mTR(Ut, R, mode),
                    oracle_sparse.ttmc_mTR(idx, vals, shape, Ut, R, mode)) < 1e-12


def test_sparse_hooi_vs_oracle(ctx, oracle_sparse, zipf_small):
    idx, vals, shape = zipf_small
    R = (8, 8, 8)
    Ut0 = _factors(shape, R, 3)
    sp = ctx.sptensor(idx, vals, shape)
    G, Ut, rep = sp.hooi(R, 3, Ut0)
    Go, Uto, res = oracle_sparse.hooi(idx, vals, shape, R, 3, Ut0)
    assert abs(rep["residual"] - res) < 1e-10
    assert abs(np.linalg.norm(G) - np.linalg.norm(Go)) < 1e-10 * np.linalg.norm(Go)
    for n in range(3):
        assert dense.principal_angle_max(Ut[n], Uto[n]) < 1e-8
        np.testing.assert_allclose(Ut[n].T @ Ut[n], np.eye(R[n]), atol=1e-12)


def test_single_nonzero_and_empty_rows(ctx, oracle_sparse):
    idx = [np.array([3], dtype=np.int64), np.array([0], dtype=np.int64),
           np.array([4], dtype=np.int64)]
    vals = np.array([2.5])
    shape = [5, 4, 6]
    R = (2, 2, 2)
    Ut = _factors(shape, R, 4)
    sp = ctx.sptensor(idx, vals, shape)
    for mode in range(3):
        Y = sp.ttmc_rows(Ut, R, mode)
        assert _rel(Y, oracle_sparse.ttmc_rows(idx, vals, shape, Ut, R, mode)) < 1e-14
        assert np.count_nonzero(np.abs(Y).sum(axis=1)) == 1


def test_out_of_range_index_is_rejected(ctx):
    from diana_tucker_b200 import DTError
    idx = [np.array([0, 5], dtype=np.int64), np.array([0, 1], dtype=np.int64)]
    with pytest.raises(DTError) as e:
        ctx.sptensor(idx, np.array([1.0, 2.0]), [5, 4])
    assert e.value.code == 1


def test_sptensor_outlives_its_context(oracle_sparse):
    """Destroying a context first detaches its sparse tensors: later calls fail
    with an error and closing the tensor is safe."""
    from diana_tucker_b200 import Context, DTError, datasets
    idx, vals, shape = datasets.sparse_zipf((50, 40, 30), 500, alpha=1.1, seed=5)
    c2 = Context(0)
    sp = c2.sptensor(idx, vals, shape)
    c2.close()
    with pytest.raises(DTError) as e:
        sp.ttmc_rows(_factors(shape, (2, 2, 2), 6), (2, 2, 2), 0)
    assert e.value.code == 1
    sp.close()
