"""The bench workloads at full size, checked through size-independent
properties (the oracle is too slow at these sizes).

Dense: the 96^4 FP32 Tucker tensor, ranks 16^4 (340 MB).
- The mixed-precision and FP64 decompositions agree on the relative error to 1e-6.
- Every factor is orthonormal to 1e-12.
- The mixed path's core equals X x_n U_n^T, recomputed here in FP64 by numpy, to
  1e-12 relative.
- The reported residual obeys res^2 = 1 - |G|^2/|X|^2 to 1e-12.

Sparse: the 2e6 x 2e5 x 5e4 tensor of 50M Zipf(1.1) draws (34.5M nonzeros), ranks 16^3.
The core G = X x_1 U_1^T x_2 U_2^T x_3 U_3^T is formed three times, once from each
mode's TTMc (Y_(n)^T U_n). The three must agree to 1e-12 relative. That exercises every
mode's fibre layout, the long-row pieces and their combine at full size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b)))


def test_dense_96x4_rank16_properties(ctx):
    from diana_tucker_b200 import DT_PREC_BF16X2, DT_PREC_FP64, datasets
    X = datasets.dense_96x4_fp32()
    R = (16, 16, 16, 16)
    kw = dict(init="randn", seed=1, max_sweeps=30, tol=1e-9)
    Gm, Um, rm = ctx.hooi_dense(X, R, precision=DT_PREC_BF16X2, inner_iters=2, **kw)
    G6, U6, r6 = ctx.hooi_dense(X, R, precision=DT_PREC_FP64, inner_iters=5, **kw)
    assert rm["sweeps"] < 30 and r6["sweeps"] < 30
    assert abs(rm["residual"] - r6["residual"]) <= 1e-6
    for U in (Um, U6):
        for u in U:
            assert np.max(np.abs(u.T @ u - np.eye(u.shape[1]))) <= 1e-12
    X64 = np.asarray(X, dtype=np.float64)
    Gc = X64
    for n in range(4):
        # Contract mode n with U_n; tensordot moves the new axis last, so after
        # four contractions the axes are back in order.
        Gc = np.tensordot(Gc, Um[n], axes=([0], [0]))
    assert _rel(Gm, Gc) <= 1e-12
    x2 = float(np.sum(X64 * X64))
    for G, rep in ((Gm, rm), (G6, r6)):
        g2 = float(np.sum(np.asarray(G) ** 2))
        assert abs(rep["residual"] ** 2 - (1.0 - g2 / x2)) <= 1e-12


def test_sparse_zipf_full_size_core_agrees_across_modes(ctx):
    from diana_tucker_b200 import datasets
    idx, vals, shape = datasets.sparse_zipf((2_000_000, 200_000, 50_000), 50_000_000,
                                            alpha=1.1, seed=2)
    R = (16, 16, 16)
    Ut = datasets.random_orthonormal_transposed(shape, R, 2)
    sp = ctx.sptensor(idx, vals, shape)
    try:
        assert sp.nnz == len(vals) > 30_000_000
        cores = []
        for mode in range(3):
            L = sp.ttmc_mTR(Ut, R, mode)  # P x R_mode = G_(mode)^T
            # Row p of L runs over the other two modes, the lower one fastest.
            A = np.asarray(L).reshape(16, 16, 16, order="F")
            cores.append({0: A.transpose(2, 0, 1), 1: A.transpose(0, 2, 1), 2: A}[mode])
    finally:
        sp.close()
    assert np.max(np.abs(cores[0])) > 0.0
    assert _rel(cores[1], cores[0]) <= 1e-12
    assert _rel(cores[2], cores[0]) <= 1e-12
