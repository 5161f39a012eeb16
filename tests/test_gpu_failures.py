"""Failure handling, with every failure made on the host or by a wait that
nothing completes: no test faults, traps or hangs the GPU.

- A bounded device wait that runs out (dt_selftest_wait_timeout: an mbarrier
  that nothing arrives on, a limit of 2e6 cycles, about 1 ms) returns
  DT_ERR_TIMEOUT; the context's next calls give the same results as before.
- A device-memory cap (dt_ctx_set_mem_limit) below a call's needs fails the
  call with DT_ERR_NOMEM before it allocates past the cap; the bytes the
  context holds come back to where they were, and lifting the cap gives the
  uncapped results bit for bit.
- NaN inputs: dense HOOI (FP64 and the tensor-core path) and sparse HOOI
  fail with DT_ERR_NUMERIC; a NaN tensor in a batch gives a NaN relative
  error for that tensor alone, the others bit-identical to a clean batch.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _codes():
    from diana_tucker_b200 import _lib
    return _lib


def _dense(shape=(40, 36, 32), seed=0):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(shape))


def test_bounded_wait_runs_out_and_context_survives(ctx):
    from diana_tucker_b200 import DTError
    L = _codes()
    X = _dense()
    G1, U1, _ = ctx.hooi_dense(X, (4, 4, 4), max_sweeps=3)
    with pytest.raises(DTError) as e:
        ctx.selftest_wait_timeout(2_000_000)
    assert e.value.code == L.DT_ERR_TIMEOUT
    # A limit above the library's own budget is refused before any launch.
    with pytest.raises(DTError) as e:
        ctx.selftest_wait_timeout(4_000_000_000)
    assert e.value.code == L.DT_ERR_ARG
    G2, U2, _ = ctx.hooi_dense(X, (4, 4, 4), max_sweeps=3)
    assert np.array_equal(G1, G2)
    for a, b in zip(U1, U2):
        assert np.array_equal(a, b)


XBYTES = 40 * 36 * 32 * 8


@pytest.mark.parametrize("tiled,cap", [(True, 1 << 20), (False, XBYTES + (16 << 10))])
def test_memory_cap_fails_cleanly_then_lifts(ctx, tiled, cap):
    """A 1.5 MB X under a 1 MiB cap fails at its staging; a 369 KB X under a
    cap of X + 16 KiB fails further into the call, in the HOOI's buffers."""
    from diana_tucker_b200 import Context, DTError
    L = _codes()
    X = _dense()
    Xc = np.asfortranarray(np.tile(X, (4, 1, 1))) if tiled else X
    Gref, Uref, _ = ctx.hooi_dense(X, (4, 4, 4), max_sweeps=3)
    c = Context(0)
    try:
        before = c.mem_usage()[0]
        c.set_mem_limit(cap)
        for _ in range(2):  # a repeated failure holds nothing more
            with pytest.raises(DTError) as e:
                c.hooi_dense(Xc, (4, 4, 4), max_sweeps=3)
            assert e.value.code == L.DT_ERR_NOMEM
            c.synchronize()
            assert c.mem_usage()[0] == before
        c.set_mem_limit(0)
        G, U, _ = c.hooi_dense(X, (4, 4, 4), max_sweeps=3)
        assert np.array_equal(G, Gref)
        for a, b in zip(U, Uref):
            assert np.array_equal(a, b)
        assert c.mem_usage()[1] > 0
    finally:
        c.close()


def test_memory_cap_on_sparse_tensor_and_tensor_core_path(ctx):
    from diana_tucker_b200 import DT_PREC_BF16XH, Context, DTError
    L = _codes()
    rng = np.random.default_rng(3)
    shape = (64, 48, 40)
    X = rng.standard_normal(shape).astype(np.float32)
    kw = dict(precision=DT_PREC_BF16XH, max_sweeps=4, tol=1e-9, inner_iters=2)
    Gref, Uref, _ = ctx.hooi_dense(X, (8, 8, 8), **kw)
    idx = [rng.integers(0, s, 5000) for s in (300, 200, 100)]
    vals = rng.standard_normal(5000)
    c = Context(0)
    try:
        c.set_mem_limit(64 << 10)
        with pytest.raises(DTError) as e:
            c.sptensor(idx, vals, (300, 200, 100))
        assert e.value.code == L.DT_ERR_NOMEM
        with pytest.raises(DTError) as e:
            c.hooi_dense(X, (8, 8, 8), **kw)
        assert e.value.code == L.DT_ERR_NOMEM
        c.set_mem_limit(0)
        G, U, _ = c.hooi_dense(X, (8, 8, 8), **kw)
        assert np.array_equal(G, Gref)
        sp = c.sptensor(idx, vals, (300, 200, 100))
        sp.close()
    finally:
        c.close()


@pytest.mark.parametrize("prec", ["FP64", "BF16XH"])
def test_nan_input_dense_hooi(ctx, prec):
    import diana_tucker_b200 as dtb
    from diana_tucker_b200 import DTError
    L = _codes()
    rng = np.random.default_rng(5)
    X = rng.standard_normal((64, 48, 40)).astype(np.float32 if prec != "FP64" else np.float64)
    X[10, 7, 3] = np.nan
    with pytest.raises(DTError) as e:
        ctx.hooi_dense(X, (8, 8, 8), max_sweeps=3, precision=getattr(dtb, "DT_PREC_" + prec),
                       inner_iters=2)
    assert e.value.code == L.DT_ERR_NUMERIC
    X[10, 7, 3] = 0.0
    G, U, rep = ctx.hooi_dense(X, (8, 8, 8), max_sweeps=3,
                               precision=getattr(dtb, "DT_PREC_" + prec), inner_iters=2)
    assert np.isfinite(rep["residual"]) and np.all(np.isfinite(G))


def test_nan_input_sparse_hooi(ctx):
    from diana_tucker_b200 import DTError, datasets
    L = _codes()
    idx, vals, shape = datasets.sparse_zipf((500, 400, 300), 20_000, seed=2)
    vals = np.array(vals, dtype=np.float64)
    vals[123] = np.nan
    R = (4, 4, 4)
    Ut0 = datasets.random_orthonormal_transposed(shape, R, 1)
    sp = ctx.sptensor(idx, vals, shape)
    try:
        with pytest.raises(DTError) as e:
            sp.hooi(R, 2, Ut0)
        assert e.value.code == L.DT_ERR_NUMERIC
    finally:
        sp.close()


def test_nan_tensor_in_a_batch_stays_in_its_slot(ctx):
    from diana_tucker_b200 import datasets
    items = datasets.batched_small(count=32, seed=9)
    rng = np.random.default_rng(109)
    U0 = [[np.linalg.qr(rng.standard_normal((X.shape[n], r[n])))[0] for n in range(3)]
          for X, r in items]
    tensors = [X.copy() for X, _ in items]
    ranks = [r for _, r in items]
    _, G1, e1, _ = ctx.hooi_batched(tensors, ranks, U0, sweeps=3, block_threads=256)
    tensors[5][1, 2, 0] = np.nan
    _, G2, e2, _ = ctx.hooi_batched(tensors, ranks, U0, sweeps=3, block_threads=256)
    assert np.isnan(e2[5])
    keep = [t for t in range(len(items)) if t != 5]
    assert np.array_equal(e1[keep], e2[keep])
    for t in keep:
        assert np.array_equal(G1[t], G2[t])
