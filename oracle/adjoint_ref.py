"""FP64 NumPy reference of the adjoint (vector-Jacobian product) of the SDP solution map.

TEST INFRASTRUCTURE ONLY: the checker for HDSDPAdjoint; never imported by the
product package. The reference solver has no adjoint, so this restates the
implicit differentiation directly from the optimality conditions
    A(X) = b,  A^T(y) + S = C,  X = N S N
(the Schur complement definition follows interface/def_hdsdp_schur.h:16-22,
the dual slack interface/hdsdp_conic_sdp.c:343-402) with FP64 linear algebra
and an explicit eigendecomposition:
    X - S = Q diag(lambda) Q^T,  Xbar = Q diag(lambda+) Q^T,  Sbar = Q diag(lambda-) Q^T
    Xhat = Q diag(x^) Q^T with x^ = lambda+ or mu/lambda- (the central point at mu)
    N = Q diag(sqrt(x^/s^)) Q^T,  M_ij = <A_i, N A_j N>
    u = g_y + A(N G_X N),  v = M^-1 u,  Z = N (A^T(v) - G_X) N
    dL/db = v,  dL/dC = Z,  dL/dA_i = -v_i Xhat - y_i Z.

The coefficients are kept as one sparse (n*n) x (m+1) matrix of vec(C), vec(A_i)
(both triangles), so the Schur matrix is assembled column by column as
    M[:, j] = Avec^T vec(N A_j N),  N A_j N = N[:, r] diag(w) N[s, :]
over the entries (r, s, w) of A_j; memory stays O(n^2 + m^2 + nnz) and the
theta layer with n = 200, m = 3,595 takes seconds.

Checked against central finite differences of the compiled reference solver
in tests/test_adjoint_cpu.py.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from oracle import kernels_ref as K


def purified_scaling(X, S, mu):
    """(N, Xhat) of the central point at mu nearest the iterate (X, S)."""
    lam, Q = np.linalg.eigh(0.5 * ((X - S) + (X - S).T))
    pos = lam > 0
    xh = np.where(pos, lam, mu / np.where(pos, 1.0, -lam))
    sh = np.where(pos, mu / np.where(pos, lam, 1.0), -lam)
    return (Q * np.sqrt(xh / sh)) @ Q.T, (Q * xh) @ Q.T


def coefficient_matrix(inst):
    """Sparse (n*n) x (m+1) matrix whose column k is vec(A_k) (column-major, both
    triangles; k = 0 is C), and per column the full entry lists (rows, cols, values)."""
    n, m = inst.n, inst.m
    col = np.repeat(np.arange(m + 1), np.diff(inst.Ap[:m + 2]))
    i, j = K.packed_to_ij(n, inst.Ai[:inst.Ap[m + 1]])
    v = np.asarray(inst.Ax[:inst.Ap[m + 1]], dtype=np.float64)
    off = i != j
    r = np.concatenate([i, j[off]])
    c = np.concatenate([j, i[off]])
    w = np.concatenate([v, v[off]])
    k = np.concatenate([col, col[off]])
    Avec = sp.csc_matrix((w, (r + c * n, k)), shape=(n * n, m + 1))
    order = np.argsort(k, kind="stable")
    starts = np.searchsorted(k[order], np.arange(m + 2))
    return Avec, (r[order], c[order], w[order], starts)


def dual_slack(inst, y, Avec=None):
    """S = C - sum_i y_i A_i (full n x n)."""
    if Avec is None:
        Avec, _ = coefficient_matrix(inst)
    s = Avec[:, 0].toarray().ravel() - Avec[:, 1:] @ np.asarray(y, dtype=np.float64)
    return s.reshape(inst.n, inst.n, order="F")


def schur_scaled(inst, N, Avec, entries):
    """M_ij = <A_i, N A_j N> for all constraints."""
    n, m = inst.n, inst.m
    r, c, w, starts = entries
    AT = Avec[:, 1:].T.tocsr()
    M = np.empty((m, m))
    for j in range(m):
        lo, hi = starts[j + 1], starts[j + 2]
        U = N[:, r[lo:hi]] @ (w[lo:hi, None] * N[c[lo:hi], :])
        M[:, j] = AT @ U.ravel(order="F")
    return 0.5 * (M + M.T)


def vjp(inst, y, X, gy, GX, mu=None):
    """Gradients (gb, gC, gAx) of L = <G_X, X> + g_y^T y at the solution (y, X)."""
    n, m = inst.n, inst.m
    Avec, entries = coefficient_matrix(inst)
    S = dual_slack(inst, y, Avec)
    if mu is None:
        # the central point at mu = <X, S>/n clipped to [1e-8, 1e-6] (the Schur matrix in
        # this scaling has a condition number near 1/mu^2, past FP64's reach below 1e-8)
        mu = min(1e-6, max(1e-8, float(np.sum(X * S)) / n))
    N, Xh = purified_scaling(X, S, mu)
    M = schur_scaled(inst, N, Avec, entries)
    T = N @ GX @ N
    u = gy + Avec[:, 1:].T @ T.ravel(order="F")
    v = np.linalg.solve(M, u)
    D = (Avec[:, 1:] @ v).reshape(n, n, order="F")
    Z = N @ (D - GX) @ N
    Z = 0.5 * (Z + Z.T)
    nnz = inst.Ap[m + 1]
    col = np.repeat(np.arange(m + 1), np.diff(inst.Ap[:m + 2]))
    i, j = K.packed_to_ij(n, inst.Ai[:nnz])
    f = np.where(i == j, 1.0, 2.0)
    yk = np.concatenate([[0.0], np.asarray(y, dtype=np.float64)])
    vk = np.concatenate([[0.0], v])
    G = np.where(col == 0, Z[i, j], -vk[col] * Xh[i, j] - yk[col] * Z[i, j])
    return v, Z, f * G
