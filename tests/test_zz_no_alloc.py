"""dt_gram_f64_noalloc (the Gram with its scratch in a fixed device array)
against dt_gram_f64, both called through the C ABI on device buffers.

Named to be collected last; it also passes alone in a fresh process (its first
call then does the one-time scratch lookup)."""
import ctypes

import numpy as np
import pytest

from diana_tucker_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative max-abs difference, as for the other FP64 Gram tests

# (shape, mode): single split, many split-K partials, and the largest mode size.
CASES = [((64, 100, 80), 0), ((40, 300, 50), 1), ((20, 20, 1024), 2), ((7, 9, 5, 6), 3)]


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).reshape(-1, order="F").copy()).cuda()


def _gram(ctx, fn, X, shape, mode):
    import torch
    I = shape[mode]
    G = torch.full((I * I,), float("nan"), dtype=torch.float64, device="cuda")
    s = (ctypes.c_int64 * len(shape))(*shape)
    torch.cuda.synchronize()
    rc = fn(ctx.h, ctypes.c_void_p(X.data_ptr()), len(shape), s, mode,
            ctypes.c_void_p(G.data_ptr()))
    _lib.check(rc)
    ctx.synchronize()
    return G.cpu().numpy().reshape((I, I), order="F")


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))


def test_noalloc_gram_matches_gram_twice(ctx):
    rng = np.random.default_rng(11)
    inputs = [(_dev(rng.standard_normal(shape)), shape, mode) for shape, mode in CASES]
    first = {}
    for rep in range(2):  # two calls in a row per case, and every case after another
        for k, (X, shape, mode) in enumerate(inputs):
            want = _gram(ctx, ctx.lib.dt_gram_f64, X, shape, mode)
            got = _gram(ctx, ctx.lib.dt_gram_f64_noalloc, X, shape, mode)
            assert np.all(np.isfinite(got))
            assert _rel(got, want) < TOL, (shape, mode, rep)
            if rep == 0:
                first[k] = got
            else:
                assert _rel(got, first[k]) < TOL, (shape, mode)


def test_noalloc_gram_rejects_oversize_and_host_buffers(ctx):
    import torch
    X = torch.zeros(1025 * 2, dtype=torch.float64, device="cuda")
    G = torch.zeros(1025 * 1025, dtype=torch.float64, device="cuda")
    s = (ctypes.c_int64 * 2)(1025, 2)
    rc = ctx.lib.dt_gram_f64_noalloc(ctx.h, ctypes.c_void_p(X.data_ptr()), 2, s, 0,
                                     ctypes.c_void_p(G.data_ptr()))
    assert rc == _lib.DT_ERR_ARG
    assert b"exceeds the limit of 1024" in ctx.lib.dt_last_error()
    Xh = np.zeros((4, 3), order="F")
    Gh = np.zeros((4, 4), order="F")
    s = (ctypes.c_int64 * 2)(4, 3)
    rc = ctx.lib.dt_gram_f64_noalloc(ctx.h, Xh.ctypes.data_as(ctypes.c_void_p), 2, s, 0,
                                     Gh.ctypes.data_as(ctypes.c_void_p))
    assert rc == _lib.DT_ERR_ARG
    assert b"device memory" in ctx.lib.dt_last_error()
