"""Batched HOOI (many small 3-way tensors in one persistent launch) vs the
FP64 oracle, tensor by tensor, from the same initial factors.

Tolerance (FP64 arithmetic in both): relative error within 1e-10, largest
principal angle between factor subspaces <= 1e-8.

The configured batch -- 4096 tensors, modes U[8,64], ranks U[2,8], 10 sweeps
-- is checked in full against the reference's own HOOI sweep (Function::ttm +
ALS_, compiled in the oracle), run tensor by tensor in a pool of spawned
processes."""
import multiprocessing as mp
import os

import numpy as np
import pytest

from oracle import dense

pytestmark = pytest.mark.gpu


def _batch(count, seed, **kw):
    from diana_tucker_b200 import datasets
    items = datasets.batched_small(count=count, seed=seed, **kw)
    rng = np.random.default_rng(seed + 100)
    U0 = [[np.linalg.qr(rng.standard_normal((X.shape[n], r[n])))[0] for n in range(3)]
          for X, r in items]
    return items, U0


def _check_vs_numpy_oracle(items, U0, U, G, relerr, sweeps=10):
    for t, (X, r) in enumerate(items):
        X64 = X.astype(np.float64)
        G2, U2, hist = dense.hooi(X64, r, sweeps, U0[t])
        res = dense.residual(np.linalg.norm(X64), np.linalg.norm(G2))
        assert abs(relerr[t] - res) < 1e-10, (t, X.shape, r)
        for n in range(3):
            assert dense.principal_angle_max(U[t][n], U2[n]) < 1e-8, (t, n)
        # The returned core is the projection of X on the returned factors.
        assert np.allclose(G[t], dense.core(X64, U[t]), rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("block", [0, 128, 512])
def test_batched_matches_oracle(ctx, block):
    items, U0 = _batch(48, 3)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    U, G, relerr, rep = ctx.hooi_batched(tensors, ranks, U0, sweeps=10, block_threads=block)
    assert rep["block_threads"] in (128, 256, 512)
    _check_vs_numpy_oracle(items, U0, U, G, relerr)


@pytest.mark.parametrize("block", [128, 256])
def test_batched_packed_small_tensors_match_oracle(ctx, block):
    """Small tensors (modes 8..24) share CTAs two and four at a time: every
    item kind (whole CTA, pairs, quads) against the oracle."""
    items, U0 = _batch(40, 11, lo=8, hi=40)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    U, G, relerr, rep = ctx.hooi_batched(tensors, ranks, U0, sweeps=6, block_threads=block)
    assert rep["pack"] == 2 and rep["items"] < len(items)
    _check_vs_numpy_oracle(items, U0, U, G, relerr, sweeps=6)


def test_batched_autotuner_and_graph_reuse(ctx):
    items, U0 = _batch(600, 5)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    U1, G1, e1, rep = ctx.hooi_batched(tensors, ranks, U0, sweeps=3, block_threads=0)
    # 600 tensors: the autotuner times every block size x packing on the whole batch.
    assert rep["candidates_timed"] >= 3
    assert 0 < rep["tune_best_ms"] <= rep["tune_worst_ms"]
    assert np.all(np.isfinite(e1)) and np.all(e1 < 1)
    U2, G2, e2, rep2 = ctx.hooi_batched(tensors, ranks, U0, sweeps=3, block_threads=0)
    assert rep2["candidates_timed"] == 0 and rep2["graph_reused"] == 1
    assert (rep2["block_threads"], rep2["pack"]) == (rep["block_threads"], rep["pack"])
    # Same inputs, same configuration: bit-identical results.
    assert np.array_equal(e1, e2)


def test_batched_rejects_oversized(ctx):
    from diana_tucker_b200 import DTError
    X = np.ones((70, 8, 8), dtype=np.float32)
    with pytest.raises(DTError) as e:
        ctx.hooi_batched([X], [(2, 2, 2)], [[np.eye(70, 2), np.eye(8, 2), np.eye(8, 2)]])
    assert e.value.code == 1


def _ref_worker(args):
    """One spawned process: the reference harness (HOOI sweep of
    hooi_als.tpp:94-114 from the given factors, 10 sweeps, no early stop) on
    a chunk of tensors.  Returns [(residual, U list)]."""
    chunk, sweeps = args
    from oracle import ref
    out = []
    for X, r, U0 in chunk:
        G, U, hist = ref.hooi_harness(np.asarray(X, dtype=np.float64), r, sweeps, 0.0, U_init=U0)
        out.append((hist[-1], U))
    return out


def test_batched_4096_configured_batch_vs_reference(ctx, oracle_ref):
    """The configured batch in one launch, every tensor against the reference."""
    items, U0 = _batch(4096, 3)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    U, G, relerr, rep = ctx.hooi_batched(tensors, ranks, U0, sweeps=10, inner_iters=5)
    assert np.all(np.isfinite(relerr))
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    nproc = max(1, min(32, os.cpu_count() or 1))
    chunks = [([(items[t][0], items[t][1], U0[t]) for t in range(i, len(items), nproc)], 10)
              for i in range(nproc)]
    with mp.get_context("spawn").Pool(nproc) as pool:
        parts = pool.map(_ref_worker, chunks)
    worst_res, worst_ang = 0.0, 0.0
    for i, part in enumerate(parts):
        for j, (res, Ur) in enumerate(part):
            t = i + j * nproc
            worst_res = max(worst_res, abs(relerr[t] - res))
            for n in range(3):
                worst_ang = max(worst_ang, dense.principal_angle_max(U[t][n], Ur[n]))
    assert worst_res <= 1e-10, worst_res
    assert worst_ang <= 1e-8, worst_ang


def test_batched_on_the_legacy_default_stream(ctx):
    """torch CUDA buffers on torch's default (legacy) stream: the launch cannot
    be captured there and runs directly, with the same results."""
    import torch
    items, U0 = _batch(24, 7)
    tensors = [X for X, _ in items]
    ranks = [r for _, r in items]
    U1, G1, e1, _ = ctx.hooi_batched(tensors, ranks, U0, sweeps=4, block_threads=256)
    pk = ctx.pack_batched(tensors, ranks, U0)
    with torch.cuda.stream(torch.cuda.default_stream()):
        Xd = torch.from_numpy(pk["X"]).cuda()
        Ud = torch.from_numpy(pk["U"]).cuda()
        Gd = torch.zeros(pk["g_size"], dtype=torch.float64, device="cuda")
        Ed = torch.zeros(pk["count"], dtype=torch.float64, device="cuda")
        rep = ctx.hooi_batched_packed(pk, Ud, Gd, Ed, X=Xd, sweeps=4, block_threads=256)
        torch.cuda.synchronize()
    assert rep["graph_reused"] == 0
    np.testing.assert_array_equal(Ed.cpu().numpy(), e1)
