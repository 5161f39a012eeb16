"""The C-ABI library builds, loads without a GPU and exports every entry point
that include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:DT_API\s+)?(?:const\s+)?[A-Za-z_0-9]+\s*\*?\s*(dt_[A-Za-z0-9_]+)\s*\(",
                            text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from diana_tucker_b200 import _lib
    from diana_tucker_b200 import build
    build.build()
    return _lib.load()


def test_header_declares_entry_points():
    names = _declared()
    for must in ["dt_ctx_create", "dt_ttm_f64", "dt_gram_f64", "dt_ttt_except_f64",
                 "dt_hooi_dense", "dt_sptensor_create", "dt_sp_ttmc_mTR", "dt_sp_ttmc_mTL",
                 "dt_sp_hooi"]:
        assert must in names


def test_every_declared_symbol_is_exported(lib):
    from diana_tucker_b200 import _lib
    for name in _declared():
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
        assert name in _lib.EXPORTED, f"{name} has no ctypes signature in _lib.py"


def test_no_gpu_context_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = lib.dt_ctx_create(0, ctypes.byref(h))
    assert rc != 0
    assert lib.dt_last_error().decode()


def test_null_arguments_are_rejected_without_a_device(lib):
    # Argument checks run before any device work.
    rc = lib.dt_ttm_f64(None, None, 3, None, 0, None, 1, None)
    assert rc == 1
    assert "dt_ctx" in lib.dt_last_error().decode()


@pytest.mark.parametrize("seed", [1, 2, 5, 20000905, 0, 2**31 + 7, 2**32 - 2])
def test_libc_rand_restatement_matches_the_c_library(lib, seed):
    """DT_INIT_RANDN_LIBC with an explicit seed draws from the library's own
    restatement of the C library's rand(); its sequence equals srand(seed)
    followed by rand() (the reference's Util::randn source), value for value."""
    import ctypes
    import numpy as np
    libc = ctypes.CDLL(None)
    libc.rand.restype = ctypes.c_int
    libc.srand.argtypes = [ctypes.c_uint]
    n = 5000
    out = np.zeros(n, dtype=np.int32)
    assert lib.dt_libc_rand_sequence(seed, n, out.ctypes.data) == 0
    libc.srand(seed)
    ref = np.array([libc.rand() for _ in range(n)], dtype=np.int32)
    assert np.array_equal(out, ref)
