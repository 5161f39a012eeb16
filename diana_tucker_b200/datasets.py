"""Seeded synthetic workloads (host numpy generation, column-major arrays).

The reference ships no datasets (its ``datasets/`` folder is git-ignored), so
every workload is generated in-process from a seed:

* ``tucker_dense``   dense Tucker product + Gaussian noise (the 200^3 FP64
  rank-10 and 96^4 FP32 rank-16 configurations, small test cases);
* ``sparse_zipf``    COO tensor with bounded-Zipf indices through a random
  permutation per mode, duplicates merged by summing, lognormal values;
* ``batched_small``  many small Tucker tensors of uneven shapes and ranks;
* ``chebyshev_family`` 256^3 tensors whose factors are orthonormalised
  mixtures of Chebyshev polynomials (the learned warm-start family).

Noise "N(0, v)" means variance v.
"""
from __future__ import annotations

import numpy as np


def _ttm(X: np.ndarray, M: np.ndarray, n: int) -> np.ndarray:
    """X x_n M for a column-major X and M of shape J x I_n."""
    Y = np.tensordot(M, X, axes=([1], [n]))  # J first
    return np.asfortranarray(np.moveaxis(Y, 0, n))


def random_orthonormal(rng: np.random.Generator, rows: int, cols: int) -> np.ndarray:
    q, _ = np.linalg.qr(rng.standard_normal((rows, cols)))
    return np.asfortranarray(q)


def tucker_dense(shape, ranks, noise_var=1e-4, seed=0, dtype=np.float64, core_decay=None,
                 return_parts=False):
    """X = G x_1 U_1 ... x_N U_N + N(0, noise_var), G ~ N(0,1) (optionally scaled
    by core_decay ** (i_1 + ... + i_N)), U_n = Q of QR of an I_n x R_n Gaussian."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    ranks = tuple(int(r) for r in ranks)
    G = np.asfortranarray(rng.standard_normal(ranks))
    if core_decay is not None:
        s = np.zeros(ranks)
        for n, r in enumerate(ranks):
            sh = [1] * len(ranks)
            sh[n] = r
            s = s + np.arange(r).reshape(sh)
        G = np.asfortranarray(G * np.power(core_decay, s))
    U = [random_orthonormal(rng, I, R) for I, R in zip(shape, ranks)]
    X = G
    for n, u in enumerate(U):
        X = _ttm(X, u, n)
    if noise_var > 0:
        noise = rng.standard_normal(X.size, dtype=np.float32 if dtype == np.float32
                                    else np.float64)
        noise = np.reshape(noise, shape, order="F") * np.sqrt(noise_var)
        X = X + noise
    X = np.asfortranarray(X.astype(dtype, copy=False))
    if return_parts:
        return X, G, U
    return X


def dense_200cube_fp64():
    """200x200x200 FP64, core 10^3 N(0,1), QR'd Gaussian factors, noise N(0,1e-4),
    seed 0 (HOOI ranks (10,10,10), HOSVD init, <= 25 sweeps or fit change < 1e-8)."""
    return tucker_dense((200, 200, 200), (10, 10, 10), noise_var=1e-4, seed=0,
                        dtype=np.float64)


def dense_96x4_fp32():
    """96^4 FP32, core 16^4 N(0,1) scaled by 0.9^(i+j+k+l), QR'd Gaussian
    factors, noise N(0,1e-6), seed 1 (HOOI ranks 16^4)."""
    return tucker_dense((96, 96, 96, 96), (16, 16, 16, 16), noise_var=1e-6, seed=1,
                        dtype=np.float32, core_decay=0.9)


def _bounded_zipf(rng, size: int, n: int, alpha: float) -> np.ndarray:
    w = np.power(np.arange(1, size + 1, dtype=np.float64), -alpha)
    cdf = np.cumsum(w)
    u = rng.random(n) * cdf[-1]
    r = np.searchsorted(cdf, u, side="right")
    return np.minimum(r, size - 1).astype(np.int64)


def sparse_zipf(shape, draws, alpha=1.1, seed=2):
    """COO tensor: per mode a bounded Zipf(alpha) rank mapped through a random
    permutation of [0, I_m); duplicate coordinates merged by summing; values
    lognormal(0, 1).  Returns (idx list of int64 arrays, vals float64, shape)."""
    rng = np.random.default_rng(seed)
    shape = [int(s) for s in shape]
    idx = []
    for I in shape:
        perm = rng.permutation(I).astype(np.int64)
        idx.append(perm[_bounded_zipf(rng, I, draws, alpha)])
    vals = rng.lognormal(0.0, 1.0, draws)
    key = np.zeros(draws, dtype=np.int64)
    mult = 1
    for m, I in enumerate(shape):
        key += idx[m] * mult
        mult *= I
    uniq, inv = np.unique(key, return_inverse=True)
    merged = np.bincount(inv, weights=vals, minlength=uniq.shape[0])
    out_idx = []
    rem = uniq.copy()
    for I in shape:
        out_idx.append((rem % I).astype(np.int64))
        rem //= I
    return out_idx, merged.astype(np.float64), shape


def sparse_2m_200k_50k():
    """2,000,000 x 200,000 x 50,000 COO from 50M draws (Zipf 1.1, lognormal),
    seed 2; sparse HOOI ranks (16,16,16)."""
    return sparse_zipf((2_000_000, 200_000, 50_000), 50_000_000, alpha=1.1, seed=2)


def random_orthonormal_transposed(shape, ranks, seed):
    """Random orthonormal factors in the reference's transposed storage
    (I_m x R_m C-contiguous = R_m x I_m col-major)."""
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(random_orthonormal(rng, I, R)) for I, R in zip(shape, ranks)]


def batched_small(count=4096, seed=3, lo=8, hi=64, rlo=2, rhi=8, noise_var=1e-4):
    """`count` 3-way FP32 Tucker tensors, modes ~ U[lo, hi], ranks ~ U[rlo, rhi]
    capped at the mode size and at the product of the other two ranks.
    Returns a list of (X, ranks)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        shape = tuple(int(v) for v in rng.integers(lo, hi + 1, size=3))
        ranks = [min(int(r), s) for r, s in zip(rng.integers(rlo, rhi + 1, size=3), shape)]
        # A Tucker model needs R_n <= prod_{m != n} R_m (else the mode-n Gram
        # has rank below R_n and the extra factor columns are arbitrary).
        for n in range(3):
            others = ranks[(n + 1) % 3] * ranks[(n + 2) % 3]
            ranks[n] = min(ranks[n], others)
        ranks = tuple(ranks)
        sub_seed = int(rng.integers(0, 2**31 - 1))
        X = tucker_dense(shape, ranks, noise_var=noise_var, seed=sub_seed, dtype=np.float32)
        out.append((X, ranks))
    return out


def chebyshev_factors(rng, size=256, degrees=24, rank=12):
    x = np.linspace(-1.0, 1.0, size)
    T = np.polynomial.chebyshev.chebvander(x, degrees - 1)  # size x degrees
    mix = rng.standard_normal((degrees, rank))
    q, _ = np.linalg.qr(T @ mix)
    return np.asfortranarray(q)


def chebyshev_family_member(seed, size=256, rank=12, decay=0.15, noise_var=1e-5,
                            dtype=np.float32, return_parts=False):
    """One tensor of the learned warm-start family (seeds 1000-2999)."""
    rng = np.random.default_rng(seed)
    U = [chebyshev_factors(rng, size, 24, rank) for _ in range(3)]
    G = rng.standard_normal((rank,) * 3)
    i = np.arange(rank)
    G = G * np.exp(-decay * (i[:, None, None] + i[None, :, None] + i[None, None, :]))
    X = np.asfortranarray(G)
    for n, u in enumerate(U):
        X = _ttm(X, u, n)
    noise = rng.standard_normal(X.size).reshape(X.shape, order="F") * np.sqrt(noise_var)
    X = np.asfortranarray((X + noise).astype(dtype))
    if return_parts:
        return X, G, U
    return X
