"""Pins the oracle before anything is checked against it (CPU only).

* The compiled reference (oracle/_ref) and the numpy restatement reproduce the
  reference's own known-answer tests TTM1 and Gram1 exactly
  (tests/testcases/function/distributed/{ttm,gram}.cpp of the reference).
* The numpy restatement agrees with the compiled reference on random inputs
  for ttm / gram / ttt_except / ALS_ / HOOI_ALS.
* The sparse C restatement agrees with the dense TTM chain of the densified
  tensor (pinned above through the reference's own Function::ttm), with a
  pure-Python loop restatement of add_outer_product_all, and with a
  pure-Python orth2.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import dense

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _ka():
    with open(os.path.join(GOLD, "ref_known_answers.json")) as f:
        return json.load(f)


def _ka_tensor(ka):
    return np.reshape(np.array(ka["tensor_colmajor"], dtype=np.float64), ka["shape"], order="F")


def test_known_answers_fixture_is_the_reference_fill():
    # FunctionDistributedTest.cpp:7-16 fills each rank's local block with
    # 10*rank + local index; the assembled global tensor holds 0..55 exactly
    # once, which the fixture text must reproduce.
    ka = _ka()
    t = np.array(ka["tensor_colmajor"])
    assert t.shape == (60,)
    assert t.min() == 0 and t.max() == 55


def test_numpy_restatement_ttm1_gram1():
    ka = _ka()
    t = _ka_tensor(ka)
    m1 = np.reshape(np.arange(16.0), (4, 4), order="F")
    m2 = np.reshape(np.arange(6.0), (2, 3), order="F")
    y = dense.ttm(dense.ttm(t, m1, 1), m2, 2)
    assert np.array_equal(y.reshape(-1, order="F"), np.array(ka["ttm1"]["expected_colmajor"]))
    g = dense.gram(t, 1)
    assert np.array_equal(g.reshape(-1, order="F"), np.array(ka["gram1"]["expected_colmajor"]))


def test_compiled_reference_ttm1_gram1(oracle_ref):
    ka = _ka()
    t = _ka_tensor(ka)
    m1 = np.reshape(np.arange(16.0), (4, 4), order="F")
    m2 = np.reshape(np.arange(6.0), (2, 3), order="F")
    y = oracle_ref.ttm(oracle_ref.ttm(t, m1, 1), m2, 2)
    assert np.array_equal(y.reshape(-1, order="F"), np.array(ka["ttm1"]["expected_colmajor"]))
    g = oracle_ref.gram(t, 1)
    assert np.array_equal(g.reshape(-1, order="F"), np.array(ka["gram1"]["expected_colmajor"]))


@pytest.mark.parametrize("shape", [(7, 6, 5), (3, 4, 5, 2), (9, 1, 4)])
def test_numpy_vs_reference_operators(oracle_ref, shape):
    rng = np.random.default_rng(1)
    X = np.asfortranarray(rng.standard_normal(shape))
    for n in range(len(shape)):
        M = np.asfortranarray(rng.standard_normal((3, shape[n])))
        np.testing.assert_allclose(dense.ttm(X, M, n), oracle_ref.ttm(X, M, n), rtol=1e-13,
                                   atol=1e-13)
        np.testing.assert_allclose(dense.gram(X, n), oracle_ref.gram(X, n), rtol=1e-13,
                                   atol=1e-12)
        bshape = tuple(2 if m == n else s for m, s in enumerate(shape))
        B = np.asfortranarray(rng.standard_normal(bshape))
        np.testing.assert_allclose(dense.ttt_except(X, B, n), oracle_ref.ttt_except(X, B, n),
                                   rtol=1e-13, atol=1e-12)


def test_numpy_vs_reference_als_and_qr(oracle_ref):
    rng = np.random.default_rng(2)
    Y = np.asfortranarray(rng.standard_normal((12, 5, 4)))
    L0, _ = np.linalg.qr(rng.standard_normal((12, 3)))
    q_ref = oracle_ref.als(Y, 0, L0, 5)
    q_np = dense.als(Y, 0, L0, 5)
    assert dense.principal_angle_max(q_ref, q_np) < 1e-12
    A = rng.standard_normal((9, 4))
    Qr, Rr = oracle_ref.reduced_qr(A)
    Qn, Rn = dense.reduced_qr(A)
    np.testing.assert_allclose(np.abs(Qr), np.abs(Qn), atol=1e-13)
    S = rng.standard_normal((5, 5)) + 5 * np.eye(5)
    np.testing.assert_allclose(oracle_ref.inverse(S), np.linalg.inv(S), rtol=1e-12, atol=1e-13)


def test_numpy_hooi_matches_reference_hooi_als(oracle_ref):
    from diana_tucker_b200 import datasets
    X = datasets.tucker_dense((20, 18, 16), (4, 3, 5), noise_var=1e-4, seed=11)
    G, U, gn, xn = oracle_ref.hooi_als(X, (4, 3, 5), 8, seed=7)
    U0 = dense.libc_randn_init(X.shape, (4, 3, 5), 7)
    G2, U2, hist = dense.hooi(X, (4, 3, 5), 8, U0)
    assert abs(gn - np.linalg.norm(G2)) <= 1e-12 * gn
    assert abs(xn - np.linalg.norm(X)) <= 1e-13 * xn
    for n in range(3):
        assert dense.principal_angle_max(U[n], U2[n]) < 1e-10


def test_reference_harness_hosvd_and_tol(oracle_ref):
    from diana_tucker_b200 import datasets
    X = datasets.tucker_dense((14, 12, 10), (3, 3, 2), noise_var=1e-3, seed=5)
    G, U, hist = oracle_ref.hooi_harness(X, (3, 3, 2), 25, 1e-12)
    U0 = dense.hosvd_init(X, (3, 3, 2))
    G2, U2, hist2 = dense.hooi(X, (3, 3, 2), 25, U0, tol=1e-12)
    assert abs(hist[-1] - hist2[-1]) < 1e-12
    for n in range(3):
        assert dense.principal_angle_max(U[n], U2[n]) < 1e-9


def test_golden_fixture_consistent_with_numpy():
    z = np.load(os.path.join(GOLD, "ref_hooi_small.npz"))
    X = z["ttm_X"]
    for n in range(3):
        np.testing.assert_allclose(dense.ttm(X, z[f"ttm_M{n}"], n), z[f"ttm_Y{n}"], rtol=1e-13,
                                   atol=1e-13)
        np.testing.assert_allclose(dense.gram(X, n), z[f"gram_{n}"], rtol=1e-13, atol=1e-12)
        np.testing.assert_allclose(dense.ttt_except(X, z[f"ttt_B{n}"], n), z[f"ttt_{n}"],
                                   rtol=1e-13, atol=1e-12)
    gn, xn = z["hooi_norms"]
    assert abs(np.linalg.norm(z["hooi_G"]) - gn) < 1e-12 * gn


# ---------------------------------------------------------------------------
# sparse restatement
# ---------------------------------------------------------------------------

def _small_sparse(seed=3, shape=(9, 7, 5), nnz=60):
    rng = np.random.default_rng(seed)
    keys = rng.choice(int(np.prod(shape)), size=nnz, replace=False)
    idx = list(np.unravel_index(keys, shape, order="F"))
    idx = [np.asarray(i, dtype=np.int64) for i in idx]
    vals = rng.lognormal(0, 1, nnz)
    return idx, vals, list(shape)


def _densify(idx, vals, shape):
    X = np.zeros(shape, order="F")
    for e in range(len(vals)):
        X[tuple(int(i[e]) for i in idx)] += vals[e]
    return X


def _py_add_outer_product_all(idx, vals, shape, Ut, R, mode):
    """Pure-Python loops over add_outer_product_all (sp_tensor.tpp:367-417):
    row i accumulates v * kron of the other factors' rows, lowest mode fastest."""
    others = [m for m in range(len(shape)) if m != mode]
    P = int(np.prod([R[m] for m in others]))
    Y = np.zeros((shape[mode], P))
    for e in range(len(vals)):
        i = int(idx[mode][e])
        for p in range(P):
            rem = p
            w = vals[e]
            for m in others:
                pm = rem % R[m]
                rem //= R[m]
                w *= Ut[m][int(idx[m][e]), pm]
            Y[i, p] += w
    return Y


def test_sparse_rows_vs_python_loops(oracle_sparse):
    idx, vals, shape = _small_sparse()
    R = [3, 2, 4]
    Ut = [np.random.default_rng(10 + m).standard_normal((shape[m], R[m])) for m in range(3)]
    for mode in range(3):
        Y = oracle_sparse.ttmc_rows(idx, vals, shape, Ut, R, mode)
        np.testing.assert_allclose(Y, _py_add_outer_product_all(idx, vals, shape, Ut, R, mode),
                                   rtol=1e-13, atol=1e-13)


def test_sparse_vs_dense_chain(oracle_sparse):
    """Y_(n) of the sparse TTMc == unfold(X x_{m != n} U_m^T, n) of the densified
    tensor, the contraction the reference's Function::ttm chain computes."""
    idx, vals, shape = _small_sparse(4, (8, 6, 7, 5), 90)
    R = [2, 3, 2, 3]
    Ut = [np.linalg.qr(np.random.default_rng(20 + m).standard_normal((shape[m], R[m])))[0]
          for m in range(4)]
    X = _densify(idx, vals, shape)
    for mode in range(4):
        Yd = X
        for m in range(4):
            if m != mode:
                Yd = dense.ttm(Yd, Ut[m].T, m)
        Yn = dense.unfold(Yd, mode)
        Ys = oracle_sparse.ttmc_rows(idx, vals, shape, Ut, R, mode)
        np.testing.assert_allclose(Ys, Yn, rtol=1e-12, atol=1e-12)
        L = oracle_sparse.ttmc_mTR(idx, vals, shape, Ut, R, mode)
        np.testing.assert_allclose(L, Yn.T @ Ut[mode], rtol=1e-12, atol=1e-12)
        out = oracle_sparse.ttmc_mTL(idx, vals, shape, Ut, R, mode, L)
        np.testing.assert_allclose(out, Yn @ L, rtol=1e-12, atol=1e-11)


def test_sparse_orth2_is_modified_gram_schmidt(oracle_sparse):
    rng = np.random.default_rng(5)
    Ut = rng.standard_normal((30, 4))  # R x I col-major == I x R row-major
    out = oracle_sparse.orth2(Ut)
    # operator_double.cpp:248-277, written out for the R rows of the R x I matrix.
    A = Ut.T.copy()
    for i in range(A.shape[0]):
        for j in range(i):
            A[i] -= A[j] * np.dot(A[i], A[j])
        A[i] /= math.sqrt(np.dot(A[i], A[i]))
    np.testing.assert_allclose(out.T, A, rtol=1e-13, atol=1e-13)


def test_sparse_hooi_matches_dense_power_sweep(oracle_sparse):
    idx, vals, shape = _small_sparse(6, (10, 9, 8), 200)
    R = [3, 3, 2]
    Ut0 = [np.linalg.qr(np.random.default_rng(30 + m).standard_normal((shape[m], R[m])))[0]
           for m in range(3)]
    G, Ut, res = oracle_sparse.hooi(idx, vals, shape, R, 3, Ut0)
    X = _densify(idx, vals, shape)
    U = [u.copy() for u in Ut0]
    for _ in range(3):
        for n in range(3):
            Y = X
            for m in range(3):
                if m != n:
                    Y = dense.ttm(Y, U[m].T, m)
            Yn = dense.unfold(Y, n)
            W = Yn @ (Yn.T @ U[n])
            q, r = np.linalg.qr(W)
            U[n] = q * np.sign(np.diag(r))
    for n in range(3):
        assert dense.principal_angle_max(Ut[n], U[n]) < 1e-10
    Gd = dense.core(X, U)
    assert abs(np.linalg.norm(G) - np.linalg.norm(Gd)) < 1e-11 * np.linalg.norm(Gd)
    assert abs(res - dense.residual(np.linalg.norm(vals), np.linalg.norm(Gd))) < 1e-11


def _with_duplicates(idx, vals, seed):
    """Repeats a few nonzeros (same coordinates, other values): the TTMc adds
    duplicates up, as add_outer_product's += does."""
    rng = np.random.default_rng(seed)
    rep = rng.choice(len(vals), size=max(1, len(vals) // 5), replace=False)
    idx = [np.concatenate([i, i[rep]]) for i in idx]
    vals = np.concatenate([vals, rng.lognormal(0, 1, rep.size)])
    return idx, vals


@pytest.mark.parametrize("shape,modes", [((9, 7, 5), []), ((9, 7, 5), [0]), ((9, 7, 5), [2, 1]),
                                         ((9, 7, 5), [0, 1, 2]), ((8, 6, 7, 5), [3, 1]),
                                         ((8, 6, 7, 5), [0, 2, 3])])
def test_sparse_ttmc_dense_vs_reference_ttm_chain(oracle_sparse, oracle_ref, shape, modes):
    """orc_sp_ttmc_dense (Function::ttmc at world size 1) == the reference's own
    Function::ttm applied to the densified tensor, one listed mode at a time."""
    idx, vals, shape = _small_sparse(7, shape, 70)
    idx, vals = _with_duplicates(idx, vals, 8)
    rng = np.random.default_rng(9)
    M = [np.asfortranarray(rng.standard_normal((3 + m, shape[m]))) for m in range(len(shape))]
    Y = oracle_sparse.ttmc_dense(idx, vals, shape, M, modes)
    Yd = _densify(idx, vals, shape)
    for m in modes:
        Yd = oracle_ref.ttm(Yd, M[m], m)
    assert Y.shape == Yd.shape
    np.testing.assert_allclose(Y, Yd, rtol=1e-12, atol=1e-12)


def test_sparse_mettmc_order_is_the_reference_sort(oracle_sparse):
    # I_m / J_m as integer quotients: 9/3 = 3, 7/4 = 1, 5/5 = 1, ascending,
    # ties in the given order.
    assert oracle_sparse.mettmc_order([9, 7, 5], [3, 4, 5], [0, 2, 1]) == [2, 1, 0]
    assert oracle_sparse.mettmc_order([9, 7, 5], [3, 4, 5], [1, 2, 0]) == [1, 2, 0]
