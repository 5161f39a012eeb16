"""Regenerates the committed golden fixtures in this folder.

1. ``ref_known_answers.json`` -- the reference's own known-answer tests, read
   as text from its test sources:
     * the global 5x4x3 input tensor that the 6-rank fixture
       (tests/testcases/function/distributed/FunctionDistributedTest.cpp:7-16)
       assembles, as printed in gram.py:5-16 (numpy order (3,4,5) = the
       column-major 5x4x3 tensor);
     * TTM1 (ttm.cpp:7-37): m1 = 4x4 with m1[i] = i, m2 = 2x3 with m2[i] = i
       (column-major), t = ttm(ttm(t, m1, 1), m2, 2), expected values
       ttm.cpp:25-32;
     * Gram1 (gram.cpp:7-19): gram(t, 1), expected values gram.cpp:12-14.
2. ``ref_hooi_small.npz`` -- outputs of the reference's own HOOI_ALS and
   Function::ttm / gram / ttt_except, run here through the compiled reference
   (oracle/_ref/libdiana_ref.so) on small seeded inputs, so GPU tests can
   compare against the reference without its sources.

Run from the repository root:  python tests/golden/make_golden.py [REF_DIR]
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _floats(text: str):
    return [float(x) for x in re.findall(r"-?\d+\.\d*|-?\d+", text)]


def known_answers(ref_dir: str) -> dict:
    d = os.path.join(ref_dir, "tests", "testcases", "function", "distributed")
    gram_py = open(os.path.join(d, "gram.py")).read()
    ttm_cpp = open(os.path.join(d, "ttm.cpp")).read()
    gram_cpp = open(os.path.join(d, "gram.cpp")).read()

    # The literal passed to tl.tensor([...]) in gram.py.
    m = re.search(r"tl\.tensor\((\[\[\[.*?\]\]\])\)", gram_py, re.S)
    t_np = np.array(_floats(m.group(1)), dtype=np.float64).reshape(3, 4, 5)
    # numpy (k, j, i) -> column-major (i, j, k): flatten in C order of the
    # (3,4,5) array is exactly the column-major data of the 5x4x3 tensor.
    t_colmajor = t_np.reshape(-1).tolist()

    ttm_gt = _floats(re.search(r"ground_truth\[\]\s*=\s*\{(.*?)\}", ttm_cpp, re.S).group(1))
    gram_gt = _floats(re.search(r"ground_truth\[\]\s*=\s*\{(.*?)\}", gram_cpp, re.S).group(1))
    return {
        "source": "reference tests/testcases/function/distributed/{gram.py,ttm.cpp,gram.cpp}",
        "shape": [5, 4, 3],
        "tensor_colmajor": t_colmajor,
        "ttm1": {
            "m1_shape": [4, 4], "m1_colmajor": list(range(16)), "mode1": 1,
            "m2_shape": [2, 3], "m2_colmajor": list(range(6)), "mode2": 2,
            "out_shape": [5, 4, 2], "expected_colmajor": ttm_gt,
        },
        "gram1": {"mode": 1, "out_shape": [4, 4], "expected_colmajor": gram_gt},
    }


def reference_runs() -> dict:
    from oracle import ref
    rng = np.random.default_rng(20240601)
    out = {}
    X = np.asfortranarray(rng.standard_normal((7, 6, 5)))
    out["ttm_X"] = X
    for n in range(3):
        M = np.asfortranarray(rng.standard_normal((3, X.shape[n])))
        out[f"ttm_M{n}"] = M
        out[f"ttm_Y{n}"] = ref.ttm(X, M, n)
        out[f"gram_{n}"] = ref.gram(X, n)
        B = np.asfortranarray(rng.standard_normal(tuple(3 if m == n else X.shape[m]
                                                        for m in range(3))))
        out[f"ttt_B{n}"] = B
        out[f"ttt_{n}"] = ref.ttt_except(X, B, n)
    # A small Tucker tensor decomposed by the reference's HOOI_ALS.
    from diana_tucker_b200 import datasets
    Xh = datasets.tucker_dense((20, 18, 16), (4, 3, 5), noise_var=1e-4, seed=11,
                               dtype=np.float64)
    G, U, gn, xn = ref.hooi_als(Xh, (4, 3, 5), 8, seed=7)
    out["hooi_X"] = Xh
    out["hooi_G"] = G
    for n in range(3):
        out[f"hooi_U{n}"] = U[n]
    out["hooi_norms"] = np.array([gn, xn])
    return out


def main():
    # The reference checkout: the first argument, else $DIANA_REF, else the
    # default location of the read-only checkout.
    ref_dir = (sys.argv[1] if len(sys.argv) > 1
               else os.environ.get("DIANA_REF", "/root/reference"))
    ka = known_answers(ref_dir)
    with open(os.path.join(HERE, "ref_known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1)
    runs = reference_runs()
    np.savez_compressed(os.path.join(HERE, "ref_hooi_small.npz"), **runs)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
