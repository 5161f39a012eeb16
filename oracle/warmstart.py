"""CPU restatement (numpy) of the learned warm start -- test infrastructure.

The warm start has no counterpart in the reference (its HOOI_ALS starts from
random factors, template/algorithm/tucker/hooi_als.tpp:74-81), so this file
restates the method's own definition; the gradients are additionally pinned
by finite differences in the tests.

  loss(E, D) = |D E U - U|_F^2 / N          U: n x N, E: k x n, D: n x k
  dL/dD = (2/N) R (E U)^T,  dL/dE = (2/N) D^T R U^T,  R = D E U - U

  init: Q = orth(D); C = X x_m Q^T for every mode; V_m = leading R_m
  eigenvectors of C_(m) C_(m)^T; U_m = Q V_m.
"""
from __future__ import annotations

import numpy as np

from . import dense


def loss_grad(U, E, D):
    U = np.asarray(U, dtype=np.float64)
    N = U.shape[1]
    H = E @ U
    R = D @ H - U
    loss = float(np.sum(R * R) / N)
    gD = (2.0 / N) * R @ H.T
    gE = (2.0 / N) * (D.T @ R) @ U.T
    return loss, gE, gD


def init(X, ranks, D):
    """Returns (U list, fit of the sketch, fit of the initial factors)."""
    X = np.asarray(X, dtype=np.float64)
    Q, _ = np.linalg.qr(np.asarray(D, dtype=np.float64))
    C = X
    for m in range(X.ndim):
        C = dense.ttm(C, Q.T, m)
    U = []
    for m in range(X.ndim):
        Cm = dense.unfold(C, m)
        w, v = np.linalg.eigh(Cm @ Cm.T)
        V = v[:, ::-1][:, : ranks[m]]
        U.append(np.asfortranarray(Q @ V))
    G = X
    for m in range(X.ndim):
        G = dense.ttm(G, U[m].T, m)
    x2 = float(np.sum(X * X))
    return U, float(np.sum(C * C)) / x2, float(np.sum(G * G)) / x2
