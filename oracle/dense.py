"""ORACLE: numpy FP64 restatement of the reference's dense HOOI path.

Test infrastructure only.  Tensors are numpy arrays in Fortran (column-major)
order, matching ``Tensor<Ty>``'s column-major strides
(template/tensor_mpi.tpp:49-53).  Unfoldings follow the reference's
``Operator::tenmat`` (template/operator/operator_cpu.tpp:56-72): the mode-n
index is the row, the remaining indices form the column with the lowest mode
varying fastest.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np


def unfold(X: np.ndarray, n: int) -> np.ndarray:
    """X_(n): I_n x prod_{m != n} I_m (operator_cpu.tpp:56-72)."""
    return np.reshape(np.moveaxis(X, n, 0), (X.shape[n], -1), order="F")


def fold(M: np.ndarray, n: int, shape) -> np.ndarray:
    """Inverse of ``unfold`` (operator_cpu.tpp:115-135)."""
    shape = list(shape)
    moved = [shape[n]] + shape[:n] + shape[n + 1:]
    return np.asfortranarray(np.moveaxis(np.reshape(M, moved, order="F"), 0, n))


def ttm(X: np.ndarray, M: np.ndarray, n: int) -> np.ndarray:
    """A x_n M with M of shape J x I_n (template/function/tensor.tpp:272-335)."""
    shape = list(X.shape)
    shape[n] = M.shape[0]
    return fold(M @ unfold(X, n), n, shape)


def gram(X: np.ndarray, n: int) -> np.ndarray:
    """A_(n) A_(n)^T (tensor.tpp:18-120)."""
    U = unfold(X, n)
    return U @ U.T


def ttt_except(A: np.ndarray, B: np.ndarray, n: int) -> np.ndarray:
    """A_(n) B_(n)^T (tensor.tpp:132-259)."""
    return unfold(A, n) @ unfold(B, n).T


def reduced_qr(A: np.ndarray):
    """Householder QR, Q of the same shape as A (matrix.tpp:86-101 ->
    LAPACK dgeqrf + dorgqr, operator_double.cpp:131-155)."""
    q, r = np.linalg.qr(A, mode="reduced")
    return q, r


def als(Y: np.ndarray, n: int, L0: np.ndarray, max_iter: int = 5) -> np.ndarray:
    """ALS_ (template/algorithm/tucker/hooi_als.tpp:7-34), step for step."""
    L = L0.copy()
    for it in range(max_iter):
        if it == 0:
            LG_inv = L
        else:
            G = L.T @ L
            LG_inv = L @ np.linalg.inv(G)
        G_invLtY = ttm(Y, LG_inv.T, n)
        YYtLG_inv = ttt_except(Y, G_invLtY, n)
        G_R = LG_inv.T @ YYtLG_inv
        L = YYtLG_inv @ np.linalg.inv(G_R)
    q, _ = reduced_qr(L)
    return q


def core(X: np.ndarray, U) -> np.ndarray:
    """G = X x_1 U_1^T ... x_N U_N^T (hooi_als.tpp:105-109)."""
    G = X
    for n, u in enumerate(U):
        G = ttm(G, u.T, n)
    return G


def residual(x_norm: float, g_norm: float) -> float:
    """sqrt(1 - ||G||^2/||A||^2) as printed by hooi_als.tpp:112-114."""
    return math.sqrt(max(0.0, 1.0 - (g_norm * g_norm) / (x_norm * x_norm)))


def hosvd_init(X: np.ndarray, ranks):
    """Leading-R_n eigenvectors of X_(n) X_(n)^T, largest first."""
    U = []
    for n, r in enumerate(ranks):
        w, v = np.linalg.eigh(gram(X, n))
        U.append(np.asfortranarray(v[:, ::-1][:, :r]))
    return U


def libc_randn_init(shape, ranks, seed: int):
    """The reference's random initial factors: srand(seed), then for each mode
    a column-major I_n x R_n block of Util::randn() draws (src/util.cpp:10-18,
    Marsaglia polar on libc rand()), orthonormalised by reduced_QR
    (hooi_als.tpp:74-81)."""
    libc = ctypes.CDLL("libc.so.6")
    libc.rand.restype = ctypes.c_int
    libc.srand(ctypes.c_uint(seed))
    RAND_MAX = 2147483647

    def randn():
        while True:
            u = (libc.rand() / RAND_MAX) * 2 - 1
            v = (libc.rand() / RAND_MAX) * 2 - 1
            r = u * u + v * v
            if not (r == 0 or r > 1):
                return u * math.sqrt(-2 * math.log(r) / r)

    U = []
    for I, R in zip(shape, ranks):
        a = np.array([randn() for _ in range(I * R)], dtype=np.float64)
        a = np.reshape(a, (I, R), order="F")
        q, _ = reduced_qr(a)
        U.append(np.asfortranarray(q))
    return U


def hooi(X: np.ndarray, ranks, max_iter: int, U0, tol: float | None = None,
         inner: int = 5):
    """HOOI_ALS sweep (hooi_als.tpp:89-122) from the given initial factors.

    With ``tol`` set, stops once two consecutive sweep residuals differ by
    less than ``tol``.  Returns (G, U, residual history)."""
    U = [np.asfortranarray(u.copy()) for u in U0]
    N = X.ndim
    x_norm = float(np.linalg.norm(X))
    hist = []
    G = None
    for _ in range(max_iter):
        for n in range(N):
            Y = X
            for i in range(N):
                if i != n:
                    Y = ttm(Y, U[i].T, i)
            U[n] = als(Y, n, U[n], inner)
        G = core(X, U)
        hist.append(residual(x_norm, float(np.linalg.norm(G))))
        if tol is not None and len(hist) >= 2 and abs(hist[-1] - hist[-2]) < tol:
            break
    if G is None:
        G = core(X, U)
    return G, U, hist


def principal_angle_max(A: np.ndarray, B: np.ndarray) -> float:
    """Largest principal angle between span(A) and span(B) (radians).

    Computed from the sine formula ||(I - Qa Qa^T) Qb||_2, which stays
    accurate for tiny angles."""
    qa, _ = np.linalg.qr(A)
    qb, _ = np.linalg.qr(B)
    resid = qb - qa @ (qa.T @ qb)
    s = np.linalg.norm(resid, 2)
    return float(math.asin(min(1.0, s)))
