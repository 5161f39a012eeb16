"""Tensor-core (tcgen05, BF16) operators and the mixed-precision HOOI vs FP64.

Tolerances (norm-wise relative error of the whole result):
  * BF16 operands:            1e-2  (unit roundoff 2^-9 per operand)
  * split hi+lo BF16 operands: 1e-4 (2^-17 per operand, FP32 accumulation)
  * mixed HOOI: residual within 1e-6 of the FP64 oracle's converged residual,
    core norm within 1e-6 relative (the final core is an FP64 projection)."""
import numpy as np
import pytest

from oracle import dense

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("shape,mode,J", [
    ((96, 96, 96), 0, 16),      # K-major A (contracted index contiguous)
    ((96, 96, 96), 2, 16),      # MN-major A, one batch
    ((96, 96, 40), 1, 16),      # MN-major A, L = 96 (partial second half), batches
    ((64, 24, 16, 8), 1, 8),    # L = 64, J < 16 (padded N)
    ((256, 17, 5), 1, 32),      # J = 32, contraction length not a multiple of 16
    ((8, 300, 7), 0, 12),       # K-major, contraction over 5 K-chunks
])
@pytest.mark.parametrize("split", [False, True])
def test_ttm_tc(ctx, shape, mode, J, split):
    rng = np.random.default_rng(abs(hash((shape, mode, J))) % 2**32)
    X = np.asfortranarray(rng.standard_normal(shape).astype(np.float32))
    U = np.asfortranarray(rng.standard_normal((shape[mode], J)))
    Y = ctx.ttm_tc(X, U, mode, split=split)
    ref = dense.ttm(X.astype(np.float64), U.T, mode)
    assert Y.shape == ref.shape
    assert _nrel(Y, ref) < (1e-4 if split else 1e-2)


@pytest.mark.parametrize("I,K", [(96, 4096), (16, 256), (128, 8192), (5, 72), (100, 64)])
@pytest.mark.parametrize("split", [False, True])
def test_gram_tc(ctx, I, K, split):
    rng = np.random.default_rng(I * 7 + K)
    Y = rng.standard_normal((I, K)).astype(np.float32)
    S = ctx.gram_tc(Y, split=split)
    Yd = Y.astype(np.float64)
    ref = Yd @ Yd.T
    assert _nrel(S, ref) < (1e-4 if split else 1e-2)
    np.testing.assert_allclose(S, S.T, rtol=0, atol=1e-6 * np.abs(ref).max())


def test_tc_unsupported_layout_is_reported(ctx):
    from diana_tucker_b200 import DTError
    X = np.ones((10, 7, 5), dtype=np.float32)  # mode 1 has L = 10 < 64
    with pytest.raises(DTError) as e:
        ctx.ttm_tc(X, np.ones((7, 4)), 1)
    assert e.value.code == 5


def test_mixed_hooi_matches_fp64_oracle(ctx):
    from diana_tucker_b200 import DT_PREC_BF16, datasets
    shape, ranks = (96, 80, 72), (8, 8, 8)
    X = datasets.tucker_dense(shape, ranks, noise_var=1e-4, seed=31, dtype=np.float32)
    G, U, rep = ctx.hooi_dense(X, ranks, init="randn", seed=5, max_sweeps=30, tol=1e-9,
                               precision=DT_PREC_BF16, refine_sweeps=2)
    assert rep["precision_used"] == DT_PREC_BF16
    X64 = X.astype(np.float64)
    U0 = dense.libc_randn_init(shape, ranks, 5)
    G2, U2, hist = dense.hooi(X64, ranks, 30, U0, tol=1e-12)
    res_ref = hist[-1]
    assert abs(rep["residual"] - res_ref) < 1e-6
    gn = float(np.linalg.norm(G2))
    assert abs(rep["g_norm"] - gn) < 1e-6 * gn
    for n in range(3):
        assert dense.principal_angle_max(U[n], U2[n]) < 1e-3
        np.testing.assert_allclose(U[n].T @ U[n], np.eye(ranks[n]), atol=1e-12)
    # The returned core is the FP64 projection of X on the returned factors.
    assert _nrel(G, dense.core(X64, U)) < 1e-12


def test_mixed_hooi_four_way_vs_fp64_gpu(ctx):
    from diana_tucker_b200 import (DT_PREC_BF16, DT_PREC_BF16X2, DT_PREC_BF16XH, DT_PREC_FP64,
                                   datasets)
    shape, ranks = (64, 64, 64, 64), (8, 8, 8, 8)
    X = datasets.tucker_dense(shape, ranks, noise_var=1e-6, seed=8, dtype=np.float32,
                              core_decay=0.9)
    _, U64, r64 = ctx.hooi_dense(X, ranks, init="randn", seed=2, max_sweeps=30, tol=1e-10,
                                 precision=DT_PREC_FP64)
    for prec in (DT_PREC_BF16, DT_PREC_BF16X2, DT_PREC_BF16XH):
        G, U, rep = ctx.hooi_dense(X, ranks, init="randn", seed=2, max_sweeps=30, tol=1e-9,
                                   precision=prec, refine_sweeps=2)
        assert rep["precision_used"] == prec
        assert abs(rep["residual"] - r64["residual"]) < 1e-6
        for n in range(4):
            assert dense.principal_angle_max(U[n], U64[n]) < 1e-3


def test_mixed_hooi_falls_back_to_fp64_outside_layout_rules(ctx):
    from diana_tucker_b200 import DT_PREC_BF16, DT_PREC_FP64, datasets
    X = datasets.tucker_dense((30, 20, 10), (3, 3, 3), noise_var=1e-4, seed=4, dtype=np.float32)
    G, U, rep = ctx.hooi_dense(X, (3, 3, 3), init="randn", seed=1, max_sweeps=4,
                               precision=DT_PREC_BF16)
    assert rep["precision_used"] == DT_PREC_FP64


@pytest.mark.parametrize("shape,ranks,prec", [
    ((128, 96, 64), (32, 16, 8), "BF16XH"),        # rank 32: the 32-column TTM tiles
    ((96, 80, 72), (12, 8, 4), "BF16X2"),          # ranks off the 16-column tile, X split
    ((64, 16, 16, 16, 16), (8, 4, 4, 4, 4), "BF16XH"),  # five modes: a three-level tree
])
def test_mixed_hooi_shapes_vs_fp64_gpu(ctx, shape, ranks, prec):
    """Uneven ranks, rank 32 and a 5-way tensor through the tensor-core HOOI:
    the converged residual within 1e-6 of the FP64 path's from the same start,
    factors within 1e-3 rad, and the core the FP64 projection of X (1e-12)."""
    import diana_tucker_b200 as dtb
    from diana_tucker_b200 import DT_PREC_FP64, datasets
    X = datasets.tucker_dense(shape, ranks, noise_var=1e-6, seed=17, dtype=np.float32)
    _, U64, r64 = ctx.hooi_dense(X, ranks, init="randn", seed=3, max_sweeps=40, tol=1e-10,
                                 precision=DT_PREC_FP64)
    p = getattr(dtb, "DT_PREC_" + prec)
    G, U, rep = ctx.hooi_dense(X, ranks, init="randn", seed=3, max_sweeps=40, tol=1e-9,
                               precision=p, inner_iters=2)
    assert rep["precision_used"] == p
    assert abs(rep["residual"] - r64["residual"]) < 1e-6
    for n in range(len(shape)):
        assert dense.principal_angle_max(U[n], U64[n]) < 1e-3, n
        np.testing.assert_allclose(U[n].T @ U[n], np.eye(ranks[n]), atol=1e-12)
    assert _nrel(G, dense.core(X.astype(np.float64), U)) < 1e-12


def test_mixed_hooi_host_input_matches_device_input(ctx):
    """A host FP32 X reaches the tensor-core path in four chunk copies, each
    rounded to BF16 as it lands; the same tensor already on the device goes
    through one rounding pass.  Shape with a ragged last chunk (658944
    elements, not a multiple of 4 x 1024): factors and core bit-identical,
    residual equal to rounding (||X||^2 is summed in another order)."""
    import torch
    from diana_tucker_b200 import DT_PREC_BF16XH, datasets
    shape, ranks = (104, 88, 72), (8, 8, 8)
    X = datasets.tucker_dense(shape, ranks, noise_var=1e-4, seed=21, dtype=np.float32)
    kw = dict(init="randn", seed=4, max_sweeps=6, tol=1e-9, precision=DT_PREC_BF16XH,
              inner_iters=2)
    Gh, Uh, rh = ctx.hooi_dense(X, ranks, **kw)  # pageable numpy memory
    flat = np.ascontiguousarray(X.reshape(-1, order="F"))
    Gp, Up, rp = ctx.hooi_dense(torch.from_numpy(flat).pin_memory(), ranks, shape=shape, **kw)
    Gd, Ud, rd = ctx.hooi_dense(torch.from_numpy(flat).cuda(), ranks, shape=shape, **kw)
    torch.cuda.synchronize()
    assert rh["sweeps"] == rp["sweeps"] == rd["sweeps"]
    for G in (Gh, Gp):
        assert np.array_equal(np.asarray(G), np.asarray(Gd))
    for U in (Uh, Up):
        for a, b in zip(U, Ud):
            assert np.array_equal(np.asarray(a), np.asarray(b))
    assert abs(rh["residual"] - rd["residual"]) < 1e-14
    assert abs(rp["residual"] - rd["residual"]) < 1e-14
