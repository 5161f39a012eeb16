"""Generates large_oracle.json and large_oracle_factors.npz: converged
reference results for the two dense benchmark tensors, computed here with the
reference's own code (oracle/_ref/libdiana_ref.so: the HOOI_ALS sweep built
from its Function::ttm and ALS_, hooi_als.tpp:94-114).

* 96^4 FP32 rank-16 (core scaled by 0.9^(i+j+k+l), noise N(0,1e-6), seed 1):
  the reference's random libc-seeded initial factors (seed 1), sweeps until
  the residual changes by less than 1e-9.  The input is upcast to FP64
  (exact).
* 200^3 FP64 rank-10 (noise N(0,1e-4), seed 0): HOSVD init, <= 25 sweeps or a
  residual change < 1e-8.

The JSON holds the residual history, ||G|| and ||X||; the .npz holds the
converged factors U_n (96 x 16 and 200 x 10, FP64), so that tests can bound
the principal angles between the GPU factors and the reference's.

Run from the repository root:  python tests/golden/make_large_oracle.py
(takes a minute or two on 8 cores).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main():
    from diana_tucker_b200 import datasets
    from oracle import dense, ref
    out = {}
    factors = {}
    X = datasets.dense_96x4_fp32().astype(np.float64)
    ranks = (16, 16, 16, 16)
    U0 = dense.libc_randn_init(X.shape, ranks, 1)
    t = time.time()
    G, U, hist = ref.hooi_harness(X, ranks, 8, 1e-9, U_init=U0)
    out["dense_96x4_r16"] = {
        "init": "libc randn + QR, seed 1", "tol": 1e-9, "sweeps": len(hist),
        "residual_hist": hist, "residual": hist[-1],
        "g_norm": float(np.linalg.norm(G)), "x_norm": float(np.linalg.norm(X)),
        "cpu_seconds": time.time() - t, "cpu_threads": os.cpu_count(),
    }
    for n, u in enumerate(U):
        factors[f"dense_96x4_r16_U{n}"] = np.asarray(u, dtype=np.float64)
    print(out["dense_96x4_r16"], flush=True)
    X1 = datasets.dense_200cube_fp64()
    t = time.time()
    G1, U1, hist1 = ref.hooi_harness(X1, (10, 10, 10), 25, 1e-8)
    out["dense_200cube_r10"] = {
        "init": "HOSVD", "tol": 1e-8, "sweeps": len(hist1), "residual_hist": hist1,
        "residual": hist1[-1], "g_norm": float(np.linalg.norm(G1)),
        "x_norm": float(np.linalg.norm(X1)), "cpu_seconds": time.time() - t,
        "cpu_threads": os.cpu_count(),
    }
    for n, u in enumerate(U1):
        factors[f"dense_200cube_r10_U{n}"] = np.asarray(u, dtype=np.float64)
    print(out["dense_200cube_r10"], flush=True)
    with open(os.path.join(HERE, "large_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "large_oracle_factors.npz"), **factors)


if __name__ == "__main__":
    main()
