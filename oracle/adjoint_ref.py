"""FP64 NumPy reference of the adjoint (vector-Jacobian product) of the SDP solution map.

TEST INFRASTRUCTURE ONLY: the checker for HDSDPAdjoint; never imported by the
product package. The reference solver has no adjoint, so this restates the
implicit differentiation directly from the optimality conditions
    A(X) = b,  A^T(y) + S = C,  X = N S N
(the Schur complement definition follows interface/def_hdsdp_schur.h:16-22,
the dual slack interface/hdsdp_conic_sdp.c:343-402) with dense NumPy
linear algebra and an explicit eigendecomposition:
    X - S = Q diag(lambda) Q^T,  Xbar = Q diag(lambda+) Q^T,  Sbar = Q diag(lambda-) Q^T
    Xhat = Q diag(x^) Q^T with x^ = lambda+ or mu/lambda- (the central point at mu)
    N = Q diag(sqrt(x^/s^)) Q^T,  M_ij = <A_i, N A_j N>
    u = g_y + A(N G_X N),  v = M^-1 u,  Z = N (A^T(v) - G_X) N
    dL/db = v,  dL/dC = Z,  dL/dA_i = -v_i Xhat - y_i Z.
Checked against central finite differences of the compiled reference solver
in tests/test_adjoint_cpu.py.
"""
from __future__ import annotations

import numpy as np

from oracle import kernels_ref as K


def purified_scaling(X, S, mu):
    """(N, Xhat) of the central point at mu nearest the iterate (X, S)."""
    lam, Q = np.linalg.eigh(0.5 * ((X - S) + (X - S).T))
    pos = lam > 0
    xh = np.where(pos, lam, mu / np.where(pos, 1.0, -lam))
    sh = np.where(pos, mu / np.where(pos, lam, 1.0), -lam)
    return (Q * np.sqrt(xh / sh)) @ Q.T, (Q * xh) @ Q.T


def vjp(inst, y, X, gy, GX, mu=None):
    """Gradients (gb, gC, gAx) of L = <G_X, X> + g_y^T y at the solution (y, X)."""
    C, A = K.dense_data(inst)
    S = K.dual_slack(C, A, y)
    if mu is None:
        # the central point at mu = <X, S>/n clipped to [1e-8, 1e-6] (the Schur matrix in
        # this scaling has a condition number near 1/mu^2, past FP64's reach below 1e-8)
        mu = min(1e-6, max(1e-8, float(np.sum(X * S)) / inst.n))
    N, Xh = purified_scaling(X, S, mu)
    m = inst.m
    NA = [N @ Ai @ N for Ai in A]
    M = np.array([[np.sum(A[i] * NA[j]) for j in range(m)] for i in range(m)])
    T = N @ GX @ N
    u = gy + np.array([np.sum(Ai * T) for Ai in A])
    v = np.linalg.solve(M, u)
    D = sum(vi * Ai for vi, Ai in zip(v, A))
    Z = N @ (D - GX) @ N
    Z = 0.5 * (Z + Z.T)
    gAx = np.zeros(inst.Ap[-1])
    for k in range(m + 1):
        lo, hi = inst.Ap[k], inst.Ap[k + 1]
        i, j = K.packed_to_ij(inst.n, inst.Ai[lo:hi])
        f = np.where(i == j, 1.0, 2.0)
        G = Z if k == 0 else (-v[k - 1] * Xh - y[k - 1] * Z)
        gAx[lo:hi] = f * G[i, j]
    return v, Z, gAx
