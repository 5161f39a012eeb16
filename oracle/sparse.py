"""ORACLE: ctypes bindings to the C restatement of the reference's sparse
Tucker path (``sparse_oracle.c``; see its header for the reference lines).

Test infrastructure only.  A sparse tensor is given as ``idx`` (ndim x nnz
int64, 0-based), ``vals`` (nnz float64) and ``shape``; factors are passed
transposed as in the reference: ``Ut[m]`` is R_m x I_m column-major, i.e. a
C-contiguous numpy array of shape (I_m, R_m) whose row i is factor row i.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libdt_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "_build/libdt_oracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_sp_fnorm.restype = ctypes.c_double
    return _lib


class _Args:
    """Keeps the ctypes pointer arrays and their numpy owners alive."""

    def __init__(self, idx, vals, shape, Ut, R):
        self.idx = [np.ascontiguousarray(i, dtype=np.int64) for i in idx]
        self.vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.shape = np.ascontiguousarray(shape, dtype=np.int64)
        self.R = np.ascontiguousarray(R, dtype=np.int64)
        self.Ut = [np.ascontiguousarray(u, dtype=np.float64) for u in Ut]
        nd = len(self.idx)
        self.idx_p = (_i64p * nd)(*[i.ctypes.data_as(_i64p) for i in self.idx])
        self.Ut_p = (_dp * nd)(*[u.ctypes.data_as(_dp) for u in self.Ut])
        self.nnz = ctypes.c_int64(self.vals.shape[0])
        self.ndim = nd


def fnorm(vals):
    v = np.ascontiguousarray(vals, dtype=np.float64)
    return lib().orc_sp_fnorm(ctypes.c_int64(v.shape[0]), v.ctypes.data_as(_dp))


def kron_len(R, mode):
    P = 1
    for m, r in enumerate(R):
        if m != mode:
            P *= int(r)
    return P


def ttmc_rows(idx, vals, shape, Ut, R, mode):
    """Y_(mode) as an I_n x P C-contiguous array."""
    a = _Args(idx, vals, shape, Ut, R)
    Y = np.zeros((int(shape[mode]), kron_len(R, mode)), dtype=np.float64)
    lib().orc_sp_ttmc_rows(a.nnz, a.ndim, a.idx_p, a.vals.ctypes.data_as(_dp),
                           a.shape.ctypes.data_as(_i64p), a.Ut_p, a.R.ctypes.data_as(_i64p),
                           mode, Y.ctypes.data_as(_dp))
    return Y


def ttmc_mTR(idx, vals, shape, Ut, R, mode):
    """L = Y_(n)^T U_n as a P x R_n Fortran-order array."""
    a = _Args(idx, vals, shape, Ut, R)
    L = np.zeros((kron_len(R, mode), int(R[mode])), dtype=np.float64, order="F")
    lib().orc_sp_ttmc_mTR(a.nnz, a.ndim, a.idx_p, a.vals.ctypes.data_as(_dp),
                          a.shape.ctypes.data_as(_i64p), a.Ut_p, a.R.ctypes.data_as(_i64p),
                          mode, L.ctypes.data_as(_dp))
    return L


def ttmc_mTL(idx, vals, shape, Ut, R, mode, L):
    """New transposed factor rows: (Y_(n) L) as an I_n x R_n C-contiguous array."""
    a = _Args(idx, vals, shape, Ut, R)
    Lf = np.asfortranarray(L, dtype=np.float64)
    out = np.zeros((int(shape[mode]), int(R[mode])), dtype=np.float64)
    lib().orc_sp_ttmc_mTL(a.nnz, a.ndim, a.idx_p, a.vals.ctypes.data_as(_dp),
                          a.shape.ctypes.data_as(_i64p), a.Ut_p, a.R.ctypes.data_as(_i64p),
                          mode, Lf.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
    return out


def orth2(Ut):
    """Modified Gram-Schmidt over the R rows of the R x I factor (in place on a copy)."""
    A = np.ascontiguousarray(Ut, dtype=np.float64).copy()
    I, R = A.shape
    lib().orc_orth2(A.ctypes.data_as(_dp), ctypes.c_int64(R), ctypes.c_int64(I))
    return A


def hooi(idx, vals, shape, R, max_iter, Ut0):
    """Sparse HOOI power sweeps from the transposed factors Ut0.
    Returns (G as P x R_{N-1} Fortran array, Ut list, residual)."""
    a = _Args(idx, vals, shape, Ut0, R)
    Ut = [u.copy() for u in a.Ut]
    Ut_p = (_dp * a.ndim)(*[u.ctypes.data_as(_dp) for u in Ut])
    last = a.ndim - 1
    G = np.zeros((kron_len(R, last), int(R[last])), dtype=np.float64, order="F")
    res = ctypes.c_double()
    lib().orc_sp_hooi(a.nnz, a.ndim, a.idx_p, a.vals.ctypes.data_as(_dp),
                      a.shape.ctypes.data_as(_i64p), a.R.ctypes.data_as(_i64p),
                      ctypes.c_int64(max_iter), Ut_p, G.ctypes.data_as(_dp), ctypes.byref(res))
    return G, Ut, res.value


def ttmc_dense(idx, vals, shape, M, idx_modes):
    """Function::ttmc(SpTensor, M, idx) at world size 1: A x_{m in idx_modes}
    M[m] (M[m] J_m x I_m) as a dense column-major array."""
    nd = len(shape)
    idx_l = [np.ascontiguousarray(i, dtype=np.int64) for i in idx]
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    shape_a = np.ascontiguousarray(shape, dtype=np.int64)
    contract = (ctypes.c_int * nd)(*[1 if m in idx_modes else 0 for m in range(nd)])
    Ms = [np.asfortranarray(M[m], dtype=np.float64) if m in idx_modes else np.zeros((1, 1))
          for m in range(nd)]
    J = np.ascontiguousarray([Ms[m].shape[0] if m in idx_modes else 0 for m in range(nd)],
                             dtype=np.int64)
    out_shape = [int(J[m]) if m in idx_modes else int(shape[m]) for m in range(nd)]
    Y = np.zeros(out_shape, dtype=np.float64, order="F")
    idx_p = (_i64p * nd)(*[i.ctypes.data_as(_i64p) for i in idx_l])
    M_p = (_dp * nd)(*[m.ctypes.data_as(_dp) for m in Ms])
    lib().orc_sp_ttmc_dense(ctypes.c_int64(vals.shape[0]), nd, idx_p, vals.ctypes.data_as(_dp),
                            shape_a.ctypes.data_as(_i64p), M_p, J.ctypes.data_as(_i64p),
                            contract, Y.ctypes.data_as(_dp))
    return Y


def mettmc_order(shape, J, idx_modes):
    """The mode order of Function::mettmc (sp_tensor.tpp:198-200): idx sorted
    by I_m / J_m (integer quotient) ascending; ties keep the given order."""
    return sorted(idx_modes, key=lambda m: int(shape[m]) // int(J[m]))
