"""The C++ drop-in API (diana_tucker_b200/cpp/include/diana) compiles against
include/dt_cuda.h and links libdt_cuda.so (CPU), and the reference's own TTM1 /
Gram1 tests written against it pass on the GPU."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "diana_tucker_b200")
OUT = os.path.join(PKG, "_build")
EXE = os.path.join(OUT, "test_dropin")


def _build():
    from diana_tucker_b200 import build
    build.build()
    os.makedirs(OUT, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(PKG, "cpp", "include"), os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp"),
           "-L", PKG, "-ldt_cuda", f"-Wl,-rpath,{PKG}", "-o", EXE]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def test_dropin_compiles_and_links():
    assert os.path.exists(_build())


@pytest.mark.gpu
def test_dropin_reference_function_tests(tmp_path):
    exe = _build()
    ka = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_known_answers.json")))
    vals = ka["tensor_colmajor"] + ka["ttm1"]["expected_colmajor"] + ka["gram1"]["expected_colmajor"]
    f = tmp_path / "ka.txt"
    f.write_text(" ".join(repr(float(v)) for v in vals))
    r = subprocess.run([exe, str(f)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ALL PASSED" in r.stdout, r.stdout + r.stderr
