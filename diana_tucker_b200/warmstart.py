"""Learned warm start for dense HOOI: family data, training and evaluation.

The method (no counterpart in the reference, whose HOOI_ALS starts from random
factors, template/algorithm/tucker/hooi_als.tpp:74-81):

* train: plain FP64 HOOI (HOSVD init, run to convergence) solves the training
  tensors; the columns of their factors train a linear autoencoder (encoder E,
  decoder D, k = 24 latent units) on the GPU with the library's own forward,
  backward and Adam kernels (``Context.ws_train``);
* infer: ``Context.ws_init`` sketches X through orth(D) in every mode (one
  pass over X), solves the small sketch's leading subspaces, refines them by
  HOOI sweeps on the sketch (the best factors inside span(D)) and decodes them
  into initial factors;
* screen and fall back: if the initial fit |X x_m U_m^T|^2 / |X|^2 is below
  the floor calibrated on the training tensors, HOSVD init is computed too
  and the better of the two starts is used;
* finish: plain HOOI from the chosen start, measured by the sweeps it needs to
  reach the converged FP64 relative error + 1e-6.

The tensor family (256^3 FP32, seeds 1000-2999): factor columns are mixtures
of the first 24 Chebyshev polynomials on [-1, 1] (random 24 x 12 Gaussian
mix, orthonormalised), core 12^3 N(0,1) * exp(-0.15 (i+j+k)), noise variance
1e-5.  Factors and core come from numpy with the tensor's seed; the Tucker
product and the noise (torch's device generator, same seed) are made on the
GPU, so a 64 MB tensor costs about a millisecond to produce.
"""
from __future__ import annotations

import time

import numpy as np

from . import DT_PREC_FP64, datasets

FAMILY = dict(size=256, rank=12, degrees=24, decay=0.15, noise_var=1e-5)


def family_member(seed: int, size: int = 256, rank: int = 12, degrees: int = 24,
                  decay: float = 0.15, noise_var: float = 1e-5, device: str = "cuda"):
    """One family tensor as a flat column-major float32 torch tensor on the
    device, plus its true factors (numpy)."""
    import torch
    rng = np.random.default_rng(seed)
    U = [datasets.chebyshev_factors(rng, size, degrees, rank) for _ in range(3)]
    G = rng.standard_normal((rank,) * 3)
    i = np.arange(rank)
    G = G * np.exp(-decay * (i[:, None, None] + i[None, :, None] + i[None, None, :]))
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)
    # Xt[k, j, i] = X[i, j, k]: C-contiguous Xt is X in column-major order.
    Xt = torch.einsum("abc,ia,jb,kc->kji", t(G), t(U[0]), t(U[1]), t(U[2]))
    if noise_var > 0:
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed))
        Xt = Xt + float(np.sqrt(noise_var)) * torch.randn(Xt.shape, generator=gen,
                                                          dtype=torch.float64, device=device)
    return Xt.to(torch.float32).reshape(-1).contiguous(), U


def first_reaching(r0: float, hist, target: float):
    """Sweeps needed to reach target: 0 if the initial residual r0 already
    does, else the 1-based sweep of the history (None if never)."""
    if r0 <= target:
        return 0
    for s, r in enumerate(hist):
        if r <= target:
            return s + 1
    return None


def solve(ctx, X, shape, ranks, *, init="hosvd", U0=None, max_sweeps=60, tol=1e-12):
    """Plain FP64 HOOI; returns (U, report)."""
    _, U, rep = ctx.hooi_dense(X, ranks, init=init, U0=U0, max_sweeps=max_sweeps, tol=tol,
                               precision=DT_PREC_FP64, want_core=False, shape=shape)
    return U, rep


def train(ctx, seeds, *, k=24, steps=600, lr=0.02, family=None, max_sweeps=60,
          sketch_sweeps=30, log=None):
    """Solves the training tensors and trains the autoencoder.  Returns a
    model dict (E, D, k, floor, loss history, timings)."""
    fam = dict(FAMILY, **(family or {}))
    n, r = fam["size"], fam["rank"]
    shape, ranks = [n] * 3, [r] * 3
    cols, fits = [], []
    t0 = time.time()
    for s in seeds:
        X, _ = family_member(s, **fam)
        U, rep = solve(ctx, X, shape, ranks, max_sweeps=max_sweeps)
        cols.extend(U)
        if log:
            log(f"train seed {s}: {rep['sweeps']} sweeps, residual {rep['residual']:.10f}")
    t_solve = time.time() - t0
    Ucols = np.asfortranarray(np.concatenate(cols, axis=1))
    t0 = time.time()
    E, D, hist = ctx.ws_train(Ucols, k, steps=steps, lr=lr, seed=7)
    t_train = time.time() - t0
    # Screening floor: the lowest initial fit over the training tensors,
    # with a 10 % margin.
    for s in seeds:
        X, _ = family_member(s, **fam)
        _, _, fi = ctx.ws_init(X, ranks, D, shape=shape, sketch_sweeps=sketch_sweeps)
        fits.append(fi)
    return dict(E=E, D=D, k=k, floor=0.9 * min(fits), loss=hist, solve_s=t_solve,
                train_s=t_train, columns=Ucols.shape[1], family=fam,
                sketch_sweeps=sketch_sweeps)


def warm_hooi(ctx, X, shape, ranks, model, *, max_sweeps=60, tol=1e-12):
    """HOOI from the learned warm start, with the HOSVD fallback.  Returns
    (U, report, info) where info has the fits and whether HOSVD was used."""
    t0 = time.time()
    U0, fs, fi = ctx.ws_init(X, ranks, model["D"], shape=shape,
                             sketch_sweeps=model.get("sketch_sweeps", 0))
    info = dict(fit_sketch=fs, fit_init=fi, screened=False, fallback=False)
    if fi < model["floor"]:
        # Suspicious start: compare with HOSVD's initial fit, keep the better.
        info["screened"] = True
        _, Uh, reph = ctx.hooi_dense(X, ranks, init="hosvd", max_sweeps=0, precision=DT_PREC_FP64,
                                     want_core=False, shape=shape)
        fh = (reph["g_norm"] / reph["x_norm"]) ** 2
        info["fit_hosvd"] = fh
        if fh > fi:
            U0 = Uh
            info["fallback"] = True
    info["init_s"] = time.time() - t0
    U, rep = solve(ctx, X, shape, ranks, init="given", U0=U0, max_sweeps=max_sweeps, tol=tol)
    return U, rep, info


def ablation_model(model, kind: str, seed: int = 11):
    """The same sketch-and-refine pipeline with another decoder, to show what
    training adds: kind "random" -- an untrained decoder (orthonormalised
    Gaussian n x k); kind "chebyshev" -- a fixed orthonormal basis of the first
    k Chebyshev polynomials on n points of [-1, 1], chosen without looking at
    any data.  The screening floor is the trained model's."""
    n, k = model["D"].shape
    if kind == "random":
        D = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, k)))[0]
    elif kind == "chebyshev":
        D = np.linalg.qr(np.polynomial.chebyshev.chebvander(np.linspace(-1.0, 1.0, n), k - 1))[0]
    else:
        raise ValueError(kind)
    return dict(model, D=np.asfortranarray(D), kind=kind)


def evaluate(ctx, seeds, model, *, max_sweeps=60, log=None, models=None):
    """Held-out comparison: sweeps and time to the converged FP64 residual +
    1e-6 (and + 1e-9), HOSVD init versus the learned warm start, and versus
    the pipeline with the decoders of `models` (name -> model; ablations)."""
    fam = model["family"]
    n, r = fam["size"], fam["rank"]
    shape, ranks = [n] * 3, [r] * 3
    rows = []
    for s in seeds:
        X, _ = family_member(s, **fam)
        t0 = time.time()
        _, rep_h = solve(ctx, X, shape, ranks, max_sweeps=max_sweeps)
        th = time.time() - t0
        t0 = time.time()
        _, rep_w, info = warm_hooi(ctx, X, shape, ranks, model, max_sweeps=max_sweeps)
        tw = time.time() - t0
        # Residual of the HOSVD start itself (evaluation only).
        _, _, rep_h0 = ctx.hooi_dense(X, ranks, init="hosvd", max_sweeps=0, precision=DT_PREC_FP64,
                                      want_core=False, want_factors=False, shape=shape)
        extra = {}
        for name, m in (models or {}).items():
            t0 = time.time()
            _, rep_a, info_a = warm_hooi(ctx, X, shape, ranks, m, max_sweeps=max_sweeps)
            extra[name] = (rep_a, info_a, time.time() - t0)
        conv = min([rep_h["residual"], rep_w["residual"]] +
                   [e[0]["residual"] for e in extra.values()])
        target = conv + 1e-6
        strict = conv + 1e-9

        def start_res(info_x):
            if info_x["fallback"]:
                return rep_h0["residual"]
            return float(np.sqrt(max(0.0, 1.0 - info_x["fit_init"])))

        r_w0 = start_res(info)
        sh = first_reaching(rep_h0["residual"], rep_h["res_hist"], target)
        sw = first_reaching(r_w0, rep_w["res_hist"], target)
        row = dict(seed=s, target=target, sweeps_hosvd=sh, sweeps_warm=sw,
                   sweeps_hosvd_strict=first_reaching(rep_h0["residual"], rep_h["res_hist"],
                                                      strict),
                   sweeps_warm_strict=first_reaching(r_w0, rep_w["res_hist"], strict),
                   wall_hosvd_s=th, wall_warm_s=tw, **info)
        for name, (rep_a, info_a, ta) in extra.items():
            ra0 = start_res(info_a)
            row[f"sweeps_{name}"] = first_reaching(ra0, rep_a["res_hist"], target)
            row[f"sweeps_{name}_strict"] = first_reaching(ra0, rep_a["res_hist"], strict)
            row[f"wall_{name}_s"] = ta
            row[f"fit_init_{name}"] = info_a["fit_init"]
            row[f"fallback_{name}"] = info_a["fallback"]
        rows.append(row)
        if log:
            log(f"eval seed {s}: hosvd {sh} sweeps, warm {sw} sweeps, fit_init {info['fit_init']:.6f}"
                f"{' (fallback)' if info['fallback'] else ''}")
    return rows


def _mean(rows, key):
    v = [r[key] for r in rows if r.get(key) is not None]
    return float(np.mean(v)) if v else None


def summarize(rows):
    ok = [r for r in rows if r["sweeps_hosvd"] is not None and r["sweeps_warm"] is not None]
    sh = np.array([r["sweeps_hosvd"] for r in ok], dtype=float)
    sw = np.array([r["sweeps_warm"] for r in ok], dtype=float)
    mh = float(sh.mean()) if len(ok) else None
    mw = float(sw.mean()) if len(ok) else None
    out = {}
    names = sorted({k[len("fit_init_"):] for r in rows for k in r if k.startswith("fit_init_")})
    for name in names:
        wall = _mean(rows, f"wall_{name}_s")
        out[name] = dict(mean_sweeps=_mean(rows, f"sweeps_{name}"),
                         mean_sweeps_strict=_mean(rows, f"sweeps_{name}_strict"),
                         mean_fit_init=_mean(rows, f"fit_init_{name}"),
                         fallback_rate=_mean(rows, f"fallback_{name}"),
                         mean_wall_ms=1e3 * wall if wall is not None else None)
    return dict(
        mean_sweeps_hosvd_strict=_mean(rows, "sweeps_hosvd_strict"),
        mean_sweeps_warm_strict=_mean(rows, "sweeps_warm_strict"),
        mean_fit_init_warm=_mean(rows, "fit_init"),
        ablation=out,
        tensors=len(rows),
        reached=len(ok),
        mean_sweeps_hosvd=mh,
        mean_sweeps_warm=mw,
        sweep_ratio=(mh / mw if mw else None) if len(ok) else None,
        mean_wall_hosvd_ms=1e3 * float(np.mean([r["wall_hosvd_s"] for r in rows])),
        mean_wall_warm_ms=1e3 * float(np.mean([r["wall_warm_s"] for r in rows])),
        fallback_rate=float(np.mean([r["fallback"] for r in rows])),
        screen_rate=float(np.mean([r["screened"] for r in rows])),
    )
