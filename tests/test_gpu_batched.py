"""Batched HOOI (many small 3-way tensors in one persistent launch) vs the
FP64 oracle, tensor by tensor, from the same initial factors.

Tolerance (FP64 arithmetic in both): relative error within 1e-10, largest
principal angle between factor subspaces <= 1e-8."""
import numpy as np
import pytest

from oracle import dense

pytestmark = pytest.mark.gpu


def _batch(count, seed):
    from diana_tucker_b200 import datasets
    items = datasets.batched_small(count=count, seed=seed)
    rng = np.random.default_rng(seed + 100)
    U0 = [[np.linalg.qr(rng.standard_normal((X.shape[n], r[n])))[0] for n in range(3)]
          for X, r in items]
    return items, U0


@pytest.mark.parametrize("block", [0, 128, 512])
def test_batched_matches_oracle(ctx, block):
    items, U0 = _batch(48, 3)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    U, G, relerr, rep = ctx.hooi_batched(tensors, ranks, U0, sweeps=10, block_threads=block)
    assert rep["block_threads"] in (128, 256, 512)
    for t, (X, r) in enumerate(items):
        X64 = X.astype(np.float64)
        G2, U2, hist = dense.hooi(X64, r, 10, U0[t])
        res = dense.residual(np.linalg.norm(X64), np.linalg.norm(G2))
        assert abs(relerr[t] - res) < 1e-10, (t, X.shape, r)
        for n in range(3):
            assert dense.principal_angle_max(U[t][n], U2[n]) < 1e-8, (t, n)
        # The returned core is the projection of X on the returned factors.
        assert np.allclose(G[t], dense.core(X64, U[t]), rtol=1e-10, atol=1e-10)


def test_batched_autotuner_reports_timings(ctx):
    items, U0 = _batch(600, 5)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    _, _, relerr, rep = ctx.hooi_batched(tensors, ranks, U0, sweeps=3, block_threads=0)
    # 600 > 512: the autotuner times three candidates on the first 512 tensors.
    assert all(v > 0 for v in rep["tune_ms"])
    assert np.all(np.isfinite(relerr)) and np.all(relerr < 1)
    _, _, _, rep2 = ctx.hooi_batched(tensors, ranks, U0, sweeps=3, block_threads=0)
    assert rep2["block_threads"] == rep["block_threads"] and rep2["tune_ms"] == [0, 0, 0]


def test_batched_rejects_oversized(ctx):
    from diana_tucker_b200 import DTError
    X = np.ones((70, 8, 8), dtype=np.float32)
    with pytest.raises(DTError) as e:
        ctx.hooi_batched([X], [(2, 2, 2)], [[np.eye(70, 2), np.eye(8, 2), np.eye(8, 2)]])
    assert e.value.code == 1
