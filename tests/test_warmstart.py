"""Learned warm start: autoencoder gradients against the CPU restatement
(oracle/warmstart.py) and finite differences, training, the sketch-based
initial factors, the HOSVD fallback, and what the trained model gains over
HOSVD init on held-out tensors of a small member of the family.

Tolerances: 1e-10 relative for FP64 kernels against the restatement (only the
summation order differs); 1e-6 relative for central differences."""
import numpy as np
import pytest

from oracle import dense
from oracle import warmstart as ows


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def _problem(seed=0, n=40, N=90, k=6):
    rng = np.random.default_rng(seed)
    U = np.asfortranarray(rng.standard_normal((n, N)))
    E = np.asfortranarray(rng.standard_normal((k, n)) / np.sqrt(n))
    D = np.asfortranarray(rng.standard_normal((n, k)) / np.sqrt(k))
    return U, E, D


def test_oracle_gradients_match_finite_differences():
    U, E, D = _problem(n=12, N=20, k=3)
    _, gE, gD = ows.loss_grad(U, E, D)
    h = 1e-6
    for P, g in ((E, gE), (D, gD)):
        num = np.zeros_like(P)
        for idx in np.ndindex(P.shape):
            old = P[idx]
            P[idx] = old + h
            lp = ows.loss_grad(U, E, D)[0]
            P[idx] = old - h
            lm = ows.loss_grad(U, E, D)[0]
            P[idx] = old
            num[idx] = (lp - lm) / (2 * h)
        assert _rel(g, num) < 1e-6


def test_oracle_init_recovers_a_span_it_was_given():
    """With D spanning the true factors, the sketch init reproduces them."""
    from diana_tucker_b200 import datasets
    rng = np.random.default_rng(5)
    U = [datasets.chebyshev_factors(rng, 40, 10, 4) for _ in range(3)]
    G = rng.standard_normal((4, 4, 4))
    X = G
    for m in range(3):
        X = dense.ttm(X, U[m], m)
    basis = np.linalg.qr(np.polynomial.chebyshev.chebvander(np.linspace(-1, 1, 40), 9))[0]
    Ui, fs, fi = ows.init(X, (4, 4, 4), basis)
    for m in range(3):
        assert dense.principal_angle_max(Ui[m], U[m]) < 1e-10
    assert abs(fi - 1.0) < 1e-12 and abs(fs - 1.0) < 1e-12


@pytest.mark.gpu
def test_loss_grad_matches_oracle(ctx):
    U, E, D = _problem()
    loss, gE, gD = ctx.ws_loss_grad(U, E, D)
    lo, gEo, gDo = ows.loss_grad(U, E, D)
    assert abs(loss - lo) <= 1e-10 * lo
    assert _rel(gE, gEo) < 1e-10
    assert _rel(gD, gDo) < 1e-10


@pytest.mark.gpu
def test_training_finds_the_column_subspace(ctx):
    """Columns drawn from a hidden 5-dim subspace: training drives the loss
    down and span(D) onto that subspace."""
    rng = np.random.default_rng(9)
    B, _ = np.linalg.qr(rng.standard_normal((48, 5)))
    U = np.asfortranarray(B @ rng.standard_normal((5, 400)))
    E, D, hist = ctx.ws_train(U, 5, steps=800, lr=0.02, seed=3)
    assert hist[-1] < 1e-6 * hist[0]
    assert dense.principal_angle_max(D, B) < 1e-4


@pytest.mark.gpu
def test_init_matches_oracle(ctx):
    from diana_tucker_b200 import datasets
    X = datasets.tucker_dense((30, 30, 30), (4, 4, 4), noise_var=1e-4, seed=11)
    rng = np.random.default_rng(2)
    D = np.asfortranarray(rng.standard_normal((30, 8)))
    U, fs, fi = ctx.ws_init(X, (4, 4, 4), D)
    Uo, fso, fio = ows.init(X, (4, 4, 4), D)
    assert abs(fs - fso) < 1e-10 and abs(fi - fio) < 1e-10
    for m in range(3):
        assert dense.principal_angle_max(U[m], Uo[m]) < 1e-8
        np.testing.assert_allclose(U[m].T @ U[m], np.eye(4), atol=1e-12)


SMALL = dict(size=96, rank=6, degrees=12, decay=0.3, noise_var=2e-4)


@pytest.fixture(scope="module")
def small_model(ctx):
    from diana_tucker_b200 import warmstart
    return warmstart.train(ctx, range(1000, 1016), k=12, steps=600, family=SMALL)


@pytest.mark.gpu
def test_warm_start_gains_over_hosvd_on_held_out(ctx, small_model):
    from diana_tucker_b200 import warmstart
    # Noisy-data HOOI factors are not exactly inside the family's span, so
    # the loss levels off well above zero.
    assert small_model["loss"][-1] < 0.1 * small_model["loss"][0]
    rows = warmstart.evaluate(ctx, range(2000, 2008), small_model)
    s = warmstart.summarize(rows)
    assert s["reached"] == len(rows)
    assert s["fallback_rate"] == 0.0
    assert s["mean_sweeps_warm"] < s["mean_sweeps_hosvd"]


@pytest.mark.gpu
def test_off_family_tensor_falls_back_to_hosvd(ctx, small_model):
    """Random (non-Chebyshev) factors: the learned span misses them, the
    initial fit falls under the floor and the HOSVD start wins."""
    import torch
    from diana_tucker_b200 import datasets, warmstart
    X = datasets.tucker_dense((96, 96, 96), (6, 6, 6), noise_var=2e-4, seed=21,
                              dtype=np.float32)
    Xd = torch.from_numpy(X.reshape(-1, order="F").copy()).cuda()
    _, rep, info = warmstart.warm_hooi(ctx, Xd, [96] * 3, [6] * 3, small_model)
    assert info["screened"] and info["fallback"]
    _, _, rep_h = ctx.hooi_dense(X, (6, 6, 6), init="hosvd", max_sweeps=60, tol=1e-12)
    assert abs(rep["residual"] - rep_h["residual"]) < 1e-9


@pytest.mark.gpu
def test_training_adds_over_an_untrained_decoder(ctx, small_model):
    """Ablation on held-out tensors: the same sketch-and-refine pipeline with
    an untrained (random orthonormal) decoder starts from a much worse fit and
    needs no fewer sweeps than the trained one; a fixed Chebyshev basis (the
    family's own generating polynomials, no training) is reported beside it."""
    from diana_tucker_b200 import warmstart
    models = {k: warmstart.ablation_model(small_model, k) for k in ("random", "chebyshev")}
    rows = warmstart.evaluate(ctx, range(2000, 2006), small_model, models=models)
    s = warmstart.summarize(rows)
    rnd, cheb = s["ablation"]["random"], s["ablation"]["chebyshev"]
    assert s["mean_fit_init_warm"] > rnd["mean_fit_init"] + 0.05
    assert s["mean_sweeps_warm"] <= rnd["mean_sweeps"]
    assert s["mean_sweeps_warm_strict"] <= rnd["mean_sweeps_strict"]
    assert cheb["mean_fit_init"] is not None and s["mean_sweeps_warm"] is not None
