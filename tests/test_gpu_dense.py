"""Dense FP64 path on the GPU vs the oracle (through the C ABI).

Tolerances: operators 1e-12 relative (FP64, different summation order);
HOOI invariants as the spec states them for the FP64 path -- relative
reconstruction error and core norm within 1e-10, largest principal angle
between factor subspaces <= 1e-8."""
import json
import os

import numpy as np
import pytest

from oracle import dense

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b)))


def test_ttm1_gram1_known_answers(ctx):
    ka = json.load(open(os.path.join(GOLD, "ref_known_answers.json")))
    t = np.reshape(np.array(ka["tensor_colmajor"]), ka["shape"], order="F")
    m1 = np.reshape(np.arange(16.0), (4, 4), order="F")
    m2 = np.reshape(np.arange(6.0), (2, 3), order="F")
    y = ctx.ttm(ctx.ttm(t, m1, 1), m2, 2)
    assert np.array_equal(y.reshape(-1, order="F"), np.array(ka["ttm1"]["expected_colmajor"]))
    g = ctx.gram(t, 1)
    assert np.array_equal(g.reshape(-1, order="F"), np.array(ka["gram1"]["expected_colmajor"]))


def test_ops_vs_reference_fixture(ctx):
    z = np.load(os.path.join(GOLD, "ref_hooi_small.npz"))
    X = z["ttm_X"]
    for n in range(3):
        assert _rel(ctx.ttm(X, z[f"ttm_M{n}"], n), z[f"ttm_Y{n}"]) < 1e-13
        assert _rel(ctx.gram(X, n), z[f"gram_{n}"]) < 1e-13
        assert _rel(ctx.ttt_except(X, z[f"ttt_B{n}"], n), z[f"ttt_{n}"]) < 1e-13


@pytest.mark.parametrize("shape,J", [
    ((200, 200, 10), 10), ((37, 19, 23), 20), ((96, 96, 96), 16), ((1, 5, 7), 3),
    ((5, 1, 7), 2), ((6, 5, 4, 3, 2), 4), ((300,), 7), ((17, 33), 33), ((4, 1000), 1),
    # Runs of 256 rows with 9..16 outputs: the FP64 tensor-core kernel, with
    # and without split contraction, with a ragged J tile.
    ((256, 40, 3), 12), ((512, 300), 16), ((16, 16, 33, 2), 9), ((256, 2, 70), 25)])
def test_ttm_shapes(ctx, shape, J):
    rng = np.random.default_rng(hash((shape, J)) % 2**32)
    X = np.asfortranarray(rng.standard_normal(shape))
    for n in range(len(shape)):
        M = np.asfortranarray(rng.standard_normal((J, shape[n])))
        assert _rel(ctx.ttm(X, M, n), dense.ttm(X, M, n)) < 1e-12


def test_ttm_device_pointers(ctx):
    import torch
    rng = np.random.default_rng(0)
    X = np.asfortranarray(rng.standard_normal((40, 30, 20)))
    M = np.asfortranarray(rng.standard_normal((8, 30)))
    # Column-major device copies: reversed-shape contiguous tensors, transposed.
    Xt = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().permute(2, 1, 0)
    Mt = torch.from_numpy(np.ascontiguousarray(M.T)).cuda().permute(1, 0)
    Y = ctx.ttm(Xt, Mt, 1)
    torch.cuda.synchronize()
    Yh = Y.permute(2, 1, 0).contiguous().cpu().numpy().T
    assert _rel(Yh, dense.ttm(X, M, 1)) < 1e-12


@pytest.mark.parametrize("shape", [(200, 100, 30), (96, 16, 16, 16), (7, 1, 9), (3, 500)])
def test_gram_and_ttt(ctx, shape):
    rng = np.random.default_rng(7)
    X = np.asfortranarray(rng.standard_normal(shape))
    for n in range(len(shape)):
        assert _rel(ctx.gram(X, n), dense.gram(X, n)) < 1e-12
        bshape = tuple(5 if m == n else s for m, s in enumerate(shape))
        B = np.asfortranarray(rng.standard_normal(bshape))
        assert _rel(ctx.ttt_except(X, B, n), dense.ttt_except(X, B, n)) < 1e-12


def test_small_linear_algebra(ctx, oracle_ref):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((50, 7))
    B = rng.standard_normal((7, 9))
    assert _rel(ctx.matmul(A, B), A @ B) < 1e-13
    C = rng.standard_normal((9, 7))
    assert _rel(ctx.matmul(A, C, transB=True), A @ C.T) < 1e-13
    D = rng.standard_normal((50, 4))
    assert _rel(ctx.matmul(A, D, transA=True), A.T @ D) < 1e-13
    Q, R = ctx.reduced_qr(A)
    Qr, Rr = oracle_ref.reduced_qr(A)
    # Same reflector convention as LAPACK: identical Q and R up to rounding.
    assert _rel(Q, Qr) < 1e-12 and _rel(R, Rr) < 1e-12
    S = rng.standard_normal((12, 12)) + 4 * np.eye(12)
    assert _rel(ctx.inverse(S), oracle_ref.inverse(S)) < 1e-11
    W = rng.standard_normal((5, 300))  # R x I, rows orthonormalised
    O = ctx.orth2(W)
    np.testing.assert_allclose(O @ O.T, np.eye(5), atol=1e-13)
    # Same row space, same triangular relation as Gram-Schmidt: W = L O.
    Lm = W @ O.T
    assert np.max(np.abs(np.triu(Lm, 1))) < 1e-12 and np.all(np.diag(Lm) > 0)


def test_inverse_singular_reports_error(ctx):
    from diana_tucker_b200 import DTError
    with pytest.raises(DTError) as e:
        ctx.inverse(np.zeros((3, 3)))
    assert e.value.code == 4


def test_als_vs_reference(ctx, oracle_ref):
    rng = np.random.default_rng(4)
    Y = np.asfortranarray(rng.standard_normal((30, 6, 5)))
    L0, _ = np.linalg.qr(rng.standard_normal((30, 4)))
    q = ctx.als(Y, 0, L0, 5)
    qr_ = oracle_ref.als(Y, 0, L0, 5)
    assert dense.principal_angle_max(q, qr_) < 1e-10
    np.testing.assert_allclose(q.T @ q, np.eye(4), atol=1e-13)


@pytest.mark.parametrize("n,r", [(96, 16), (97, 13), (150, 16), (200, 10), (256, 8), (64, 32),
                                 (40, 20), (5, 5), (33, 1), (300, 12)])
def test_als_subspace_sizes_vs_oracle(ctx, n, r):
    """dt_als_f64 over the subspace kernel's shapes: S staged whole, packed, or
    read from L2; ranks padded to 8, 16 and 32; n above the tiled kernel's 256."""
    rng = np.random.default_rng(n * 100 + r)
    Y = np.asfortranarray(rng.standard_normal((n, 12, max(4, (2 * n) // 12 + 1))))
    L0, _ = np.linalg.qr(rng.standard_normal((n, r)))
    q = ctx.als(Y, 0, L0, 5)
    want = dense.als(Y, 0, L0, 5)
    assert dense.principal_angle_max(q, want) < 1e-10
    np.testing.assert_allclose(q.T @ q, np.eye(r), atol=1e-13)


def _check_hooi(G, U, rep, gn_ref, U_ref, xn):
    assert abs(rep["g_norm"] - gn_ref) <= 1e-10 * gn_ref
    assert abs(np.linalg.norm(G) - gn_ref) <= 1e-10 * gn_ref
    assert abs(rep["x_norm"] - xn) <= 1e-12 * xn
    res_ref = dense.residual(xn, gn_ref)
    assert abs(rep["residual"] - res_ref) <= 1e-10
    for n in range(len(U)):
        assert dense.principal_angle_max(U[n], U_ref[n]) <= 1e-8
        np.testing.assert_allclose(U[n].T @ U[n], np.eye(U[n].shape[1]), atol=1e-12)


def test_hooi_dropin_vs_reference_fixture(ctx):
    """HOOI_ALS semantics (libc-seeded random init, fixed sweeps) against the
    reference's own HOOI_ALS output stored in the golden fixture."""
    z = np.load(os.path.join(GOLD, "ref_hooi_small.npz"))
    X = z["hooi_X"]
    G, U, rep = ctx.hooi_dense(X, (4, 3, 5), init="randn", seed=7, max_sweeps=8)
    gn, xn = z["hooi_norms"]
    _check_hooi(G, U, rep, gn, [z[f"hooi_U{n}"] for n in range(3)], xn)
    assert rep["sweeps"] == 8


def test_hooi_dropin_vs_live_reference(ctx, oracle_ref):
    from diana_tucker_b200 import datasets
    X = datasets.tucker_dense((30, 25, 20, 12), (5, 4, 3, 2), noise_var=1e-3, seed=21)
    Gr, Ur, gn, xn = oracle_ref.hooi_als(X, (5, 4, 3, 2), 6, seed=3)
    G, U, rep = ctx.hooi_dense(X, (5, 4, 3, 2), init="randn", seed=3, max_sweeps=6)
    _check_hooi(G, U, rep, gn, Ur, xn)


def test_hooi_200cube_hosvd_tol_vs_reference_harness(ctx, oracle_ref):
    """The 200^3 FP64 rank-(10,10,10) configuration: HOSVD init, <= 25 sweeps or
    residual change < 1e-8, against the reference-built harness."""
    from diana_tucker_b200 import datasets
    X = datasets.dense_200cube_fp64()
    Gr, Ur, hist = oracle_ref.hooi_harness(X, (10, 10, 10), 25, 1e-8)
    G, U, rep = ctx.hooi_dense(X, (10, 10, 10), init="hosvd", max_sweeps=25, tol=1e-8)
    xn = float(np.linalg.norm(X))
    _check_hooi(G, U, rep, float(np.linalg.norm(Gr)), Ur, xn)
    assert abs(rep["residual"] - hist[-1]) <= 1e-10


@pytest.mark.parametrize("shape,ranks", [((24, 20, 16), (4, 4, 3)),
                                         ((16, 16, 48), (12, 12, 10))])
def test_hooi_fp32_input_equals_upcast(ctx, shape, ranks):
    from diana_tucker_b200 import datasets
    X32 = datasets.tucker_dense(shape, ranks, noise_var=1e-4, seed=9, dtype=np.float32)
    G1, U1, r1 = ctx.hooi_dense(X32, ranks, init="hosvd", max_sweeps=5)
    G2, U2, r2 = ctx.hooi_dense(X32.astype(np.float64), ranks, init="hosvd", max_sweeps=5)
    assert abs(r1["g_norm"] - r2["g_norm"]) <= 1e-12 * r2["g_norm"]
    for n in range(3):
        assert dense.principal_angle_max(U1[n], U2[n]) < 1e-10


def test_hooi_given_init_and_zero_sweeps(ctx):
    from diana_tucker_b200 import datasets
    X = datasets.tucker_dense((15, 14, 13), (3, 3, 3), noise_var=1e-4, seed=2)
    rng = np.random.default_rng(0)
    U0 = [np.linalg.qr(rng.standard_normal((s, 3)))[0] for s in X.shape]
    G, U, rep = ctx.hooi_dense(X, (3, 3, 3), U0=U0, max_sweeps=0)
    Gd = dense.core(X, U0)
    assert _rel(G, Gd) < 1e-12
    G, U, rep = ctx.hooi_dense(X, (3, 3, 3), U0=U0, max_sweeps=4)
    G2, U2, hist = dense.hooi(X, (3, 3, 3), 4, U0)
    assert abs(rep["g_norm"] - np.linalg.norm(G2)) < 1e-10 * np.linalg.norm(G2)


def test_hooi_rejects_bad_ranks(ctx):
    from diana_tucker_b200 import DTError
    with pytest.raises(DTError) as e:
        ctx.hooi_dense(np.ones((4, 5, 6)), (5, 2, 2))
    assert e.value.code == 1
