"""ORACLE: ctypes bindings to the reference's own dense HOOI code.

Test infrastructure only.  ``_ref/libdiana_ref.so`` is compiled in place from
the reference sources by ``oracle/Makefile`` (see ``ref_harness.cpp`` for the
reference routine behind each entry point).  All arrays are FP64 numpy arrays
in Fortran order.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libdiana_ref.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"compiled reference oracle missing: {LIB_PATH} "
                               "(run `make -C oracle` where the reference sources exist)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.ref_fnorm.restype = ctypes.c_double
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _shape(shape):
    return np.ascontiguousarray(np.asarray(shape, dtype=np.int64))


def _f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def ttm(X, M, n):
    X = _f64(X)
    M = _f64(M)
    shape = list(X.shape)
    out_shape = shape.copy()
    out_shape[n] = M.shape[0]
    Y = np.zeros(out_shape, dtype=np.float64, order="F")
    s = _shape(shape)
    lib().ref_ttm(_d(X), len(shape), s.ctypes.data_as(_i64p), n, _d(M),
                  ctypes.c_int64(M.shape[0]), _d(Y))
    return Y


def gram(X, n):
    X = _f64(X)
    G = np.zeros((X.shape[n], X.shape[n]), dtype=np.float64, order="F")
    s = _shape(X.shape)
    lib().ref_gram(_d(X), X.ndim, s.ctypes.data_as(_i64p), n, _d(G))
    return G


def ttt_except(A, B, n):
    A = _f64(A)
    B = _f64(B)
    C = np.zeros((A.shape[n], B.shape[n]), dtype=np.float64, order="F")
    sa, sb = _shape(A.shape), _shape(B.shape)
    lib().ref_ttt_except(_d(A), sa.ctypes.data_as(_i64p), _d(B), sb.ctypes.data_as(_i64p),
                         A.ndim, n, _d(C))
    return C


def reduced_qr(A):
    A = _f64(A)
    m, k = A.shape
    Q = np.zeros((m, k), dtype=np.float64, order="F")
    R = np.zeros((k, k), dtype=np.float64, order="F")
    lib().ref_reduced_qr(_d(A), ctypes.c_int64(m), ctypes.c_int64(k), _d(Q), _d(R))
    return Q, R


def inverse(A):
    A = _f64(A)
    out = np.zeros_like(A, order="F")
    lib().ref_inverse(_d(A), ctypes.c_int64(A.shape[0]), _d(out))
    return out


def fnorm(X):
    X = _f64(X)
    s = _shape(X.shape)
    return lib().ref_fnorm(_d(X), X.ndim, s.ctypes.data_as(_i64p))


def als(Y, n, L0, max_iter=5):
    Y = _f64(Y)
    L0 = _f64(L0)
    Q = np.zeros_like(L0, order="F")
    s = _shape(Y.shape)
    lib().ref_als(_d(Y), Y.ndim, s.ctypes.data_as(_i64p), n, _d(L0),
                  ctypes.c_int64(L0.shape[1]), ctypes.c_int64(max_iter), _d(Q))
    return Q


def hooi_als(X, ranks, max_iter, seed):
    """The reference's HOOI_ALS (random init from srand(seed)).
    Returns (G, U, ||G||, ||X||)."""
    X = _f64(X)
    N = X.ndim
    G = np.zeros(tuple(ranks), dtype=np.float64, order="F")
    U = [np.zeros((X.shape[n], ranks[n]), dtype=np.float64, order="F") for n in range(N)]
    Uptr = (_dp * N)(*[_d(u) for u in U])
    gn = ctypes.c_double()
    xn = ctypes.c_double()
    s = _shape(X.shape)
    r = _shape(ranks)
    lib().ref_hooi_als(_d(X), N, s.ctypes.data_as(_i64p), r.ctypes.data_as(_i64p),
                       ctypes.c_int64(max_iter), ctypes.c_uint(seed), _d(G), Uptr,
                       ctypes.byref(gn), ctypes.byref(xn))
    return G, U, gn.value, xn.value


def hooi_als_mt(X, ranks, max_iter, seed, threads=0):
    """The reference's HOOI_ALS on `threads` OpenMP threads (0: all), as it
    runs in production; the random start then varies run to run.
    Returns (||G||, ||X||)."""
    X = _f64(X)
    gn = ctypes.c_double()
    xn = ctypes.c_double()
    s = _shape(X.shape)
    r = _shape(ranks)
    lib().ref_hooi_als_mt(_d(X), X.ndim, s.ctypes.data_as(_i64p), r.ctypes.data_as(_i64p),
                          ctypes.c_int64(max_iter), ctypes.c_uint(seed), ctypes.c_int(threads),
                          ctypes.byref(gn), ctypes.byref(xn))
    return gn.value, xn.value


def hooi_harness(X, ranks, max_iter, tol, U_init=None):
    """HOOI sweep built from the reference's Function::ttm + ALS_ with HOSVD
    init (U_init None) or the given factors, stopping on residual change < tol.
    Returns (G, U, residual history)."""
    X = _f64(X)
    N = X.ndim
    G = np.zeros(tuple(ranks), dtype=np.float64, order="F")
    U = [np.zeros((X.shape[n], ranks[n]), dtype=np.float64, order="F") for n in range(N)]
    Uptr = (_dp * N)(*[_d(u) for u in U])
    if U_init is None:
        init_ptr = None
        keep = None
    else:
        keep = [_f64(u) for u in U_init]
        init_ptr = (_dp * N)(*[_d(u) for u in keep])
    hist = np.zeros(max_iter, dtype=np.float64)
    s = _shape(X.shape)
    r = _shape(ranks)
    sweeps = lib().ref_hooi_harness(_d(X), N, s.ctypes.data_as(_i64p), r.ctypes.data_as(_i64p),
                                    ctypes.c_int64(max_iter), ctypes.c_double(tol),
                                    1 if U_init is None else 0, init_ptr, _d(G), Uptr, _d(hist))
    return G, U, list(hist[:sweeps])


def read_tns(path):
    """read_data<double> (src/read_data.cpp:36-129): (idx list of 0-based int64
    arrays, vals, dims)."""
    L = lib()
    nd, nz = ctypes.c_int64(), ctypes.c_int64()
    L.ref_read_tns(path.encode(), ctypes.byref(nd), ctypes.byref(nz))
    dims = np.zeros(nd.value, dtype=np.int64)
    idx = np.zeros(nd.value * nz.value, dtype=np.int64)
    vals = np.zeros(nz.value)
    L.ref_read_tns_copy(dims.ctypes.data_as(_i64p), idx.ctypes.data_as(_i64p), _d(vals))
    return [idx[m * nz.value:(m + 1) * nz.value] for m in range(nd.value)], vals, dims
