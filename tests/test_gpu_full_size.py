"""The bench workloads at full size.

Dense: the 96^4 FP32 Tucker tensor, ranks 16^4 (340 MB).
- The FP64 path, from the reference's libc-seeded initial factors (seed 1),
  against the reference's own converged HOOI (tests/golden/large_oracle.json and
  large_oracle_factors.npz, made by make_large_oracle.py with the reference
  compiled in the oracle): residual and ||G|| within 1e-10, every principal
  angle <= 1e-8.
- The mixed-precision path against the same reference: residual and ||G||
  within 1e-6 (the method's target), principal angles <= 1e-4.
- Every factor is orthonormal to 1e-12; the mixed path's core equals
  X x_n U_n^T, recomputed here in FP64 by numpy, to 1e-12 relative; the
  reported residual obeys res^2 = 1 - |G|^2/|X|^2 to 1e-12.

Sparse: the 2e6 x 2e5 x 5e4 tensor of 50M Zipf(1.1) draws (34.5M nonzeros),
ranks 16^3.
- ttmc_mTR of every mode against the C restatement of the reference's TTMc
  (oracle/sparse_oracle.c, OpenMP), at 1e-12 relative: every mode's fibre
  layout, the long-row pieces and their two-level combine, at full size.
- The core G = X x_1 U_1^T x_2 U_2^T x_3 U_3^T formed from each mode's TTMc
  agrees across the three modes to 1e-12.
"""
import json
import os

import numpy as np
import pytest

from oracle import dense

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b)))


def _ref_96x4():
    with open(os.path.join(GOLD, "large_oracle.json")) as f:
        d = json.load(f)["dense_96x4_r16"]
    z = np.load(os.path.join(GOLD, "large_oracle_factors.npz"))
    return d, [z[f"dense_96x4_r16_U{n}"] for n in range(4)]


@pytest.fixture(scope="module")
def x96():
    from diana_tucker_b200 import datasets
    return datasets.dense_96x4_fp32()


def test_dense_96x4_fp64_vs_reference(ctx, x96):
    """The drop-in FP64 path (X as Tensor<double>, five ALS_ steps per mode)
    reproduces the reference's converged decomposition."""
    from diana_tucker_b200 import DT_PREC_FP64
    ref, Uref = _ref_96x4()
    X = x96.astype(np.float64)
    G, U, rep = ctx.hooi_dense(X, (16,) * 4, init="randn", seed=1, max_sweeps=30, tol=1e-9,
                               precision=DT_PREC_FP64, inner_iters=5)
    assert rep["sweeps"] == ref["sweeps"]
    assert abs(rep["residual"] - ref["residual"]) <= 1e-10
    assert abs(rep["g_norm"] - ref["g_norm"]) <= 1e-10 * ref["g_norm"]
    assert abs(float(np.linalg.norm(G)) - ref["g_norm"]) <= 1e-10 * ref["g_norm"]
    assert abs(rep["x_norm"] - ref["x_norm"]) <= 1e-12 * ref["x_norm"]
    for n in range(4):
        assert dense.principal_angle_max(U[n], Uref[n]) <= 1e-8, n


@pytest.mark.parametrize("prec", ["BF16X2", "BF16XH"])
def test_dense_96x4_mixed_vs_reference(ctx, x96, prec):
    import diana_tucker_b200 as dtb
    ref, Uref = _ref_96x4()
    G, U, rep = ctx.hooi_dense(x96, (16,) * 4, init="randn", seed=1, max_sweeps=30, tol=1e-9,
                               precision=getattr(dtb, "DT_PREC_" + prec), inner_iters=2)
    assert rep["sweeps"] < 30
    assert abs(rep["residual"] - ref["residual"]) <= 1e-6
    assert abs(rep["g_norm"] - ref["g_norm"]) <= 1e-6 * ref["g_norm"]
    for n in range(4):
        assert dense.principal_angle_max(U[n], Uref[n]) <= 1e-4, n


def test_dense_96x4_rank16_properties(ctx, x96):
    from diana_tucker_b200 import DT_PREC_BF16X2, DT_PREC_FP64
    X = x96
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


@pytest.fixture(scope="module")
def zipf_full():
    from diana_tucker_b200 import datasets
    idx, vals, shape = datasets.sparse_2m_200k_50k()
    R = (16, 16, 16)
    Ut = datasets.random_orthonormal_transposed(shape, R, 2)
    return idx, vals, shape, R, Ut


def test_sparse_zipf_full_size_mTR_vs_oracle(ctx, zipf_full, oracle_sparse):
    """Every mode's TTMc (Y_(n)^T U_n) at 34.5M nonzeros against the C oracle."""
    idx, vals, shape, R, Ut = zipf_full
    sp = ctx.sptensor(idx, vals, shape)
    try:
        assert sp.nnz == len(vals) > 30_000_000
        for mode in range(3):
            L = sp.ttmc_mTR(Ut, R, mode)
            Lo = oracle_sparse.ttmc_mTR(idx, vals, shape, Ut, R, mode)
            assert np.max(np.abs(Lo)) > 0.0
            assert _rel(L, Lo) <= 1e-12, mode
    finally:
        sp.close()


def test_sparse_zipf_full_size_core_agrees_across_modes(ctx, zipf_full):
    idx, vals, shape, R, Ut = zipf_full
    sp = ctx.sptensor(idx, vals, shape)
    try:
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
