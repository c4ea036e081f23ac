"""NumPy restatement of the reference's per-iteration kernels (FP64).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker for the GPU kernels;
never imported by the product package. Pinned against golden vectors dumped
from the compiled reference (tests/golden/, generated by
tests/golden/make_golden.py through oracle/ref_probe.c).

Restated formulas (reference file:line):
  dual slack      S = dC*C + dA*sum_i w_i A_i + dEye*I
                  interface/hdsdp_conic_sdp.c:343-402 (sdpDenseConeIUpdateBuffer)
  Schur matrix    M_ij = <A_i, S^-1 A_j S^-1>
                  interface/def_hdsdp_schur.h:16-22, strategies M2-M5 at
                  interface/hdsdp_conic_sdp.c:683-981
  RHS vectors     ASinv_i = <A_i, S^-1>,  ASinvRdSinv_i = r <A_i, S^-2>,
                  trace(S^-1) (only when r != 0)
                  interface/hdsdp_conic_sdp.c:746-752, :1756-1760
  log barrier     log det S = 2 sum log L_ii    interface/hdsdp_conic_sdp.c:2185-2224
  step bound      max alpha with S + alpha dS psd (the reference estimates it with
                  Lanczos, linalg/hdsdp_lanczos.c:161-292; this is the exact value)
  primal recovery X = mu (S^-1 + S^-1 (A^* dy) S^-1)
                  interface/hdsdp_conic_sdp.c:2328-2379
"""
from __future__ import annotations

import numpy as np


def packed_to_ij(n: int, rows):
    """(i, j), i >= j, of packed lower-triangle (column-major) indices (hdsdp_utils.h:49)."""
    rows = np.asarray(rows, dtype=np.int64)
    starts = np.array([(2 * n - j - 1) * j // 2 + j for j in range(n)], dtype=np.int64)
    j = np.searchsorted(starts, rows, side="right") - 1
    i = rows - starts[j] + j
    return i, j


def unpack_column(n: int, rows, vals) -> np.ndarray:
    """Full symmetric matrix from packed lower-triangle entries."""
    i, j = packed_to_ij(n, rows)
    vals = np.asarray(vals, dtype=np.float64)
    M = np.zeros((n, n))
    M[i, j] += vals
    off = i != j
    M[j[off], i[off]] += vals[off]
    return M


def rank_one_factor(n: int, rows, vals) -> np.ndarray:
    """a with A = a a^T for a packed positive rank-one column (first support entry positive)."""
    i, j = packed_to_ij(n, rows)
    vals = np.asarray(vals, dtype=np.float64)
    s0 = j.min()
    a = np.zeros(n)
    d = vals[(i == j)]
    a[i[i == j]] = np.sqrt(d)
    col = j == s0
    a[i[col]] = np.sign(vals[col]) * a[i[col]]
    return a


def dense_data(inst):
    """(C, [A_1..A_m]) as dense symmetric matrices (small n only)."""
    C = unpack_column(inst.n, *inst.column(0))
    A = [unpack_column(inst.n, *inst.column(k)) for k in range(1, inst.m + 1)]
    return C, A


def dual_slack(C, A, w, dC=1.0, dA=-1.0, dEye=0.0):
    S = dC * C + dEye * np.eye(C.shape[0])
    for wi, Ai in zip(w, A):
        if wi != 0.0:
            S = S + dA * wi * Ai
    return S


def schur(C, A, y, resi):
    """Reference KKT build at S = C - A^T y - resi I (KKT_TYPE_INFEASIBLE)."""
    S = dual_slack(C, A, y, 1.0, -1.0, -resi)
    W = np.linalg.inv(S)
    W = 0.5 * (W + W.T)
    m = len(A)
    WAW = [W @ Ai @ W for Ai in A]
    M = np.zeros((m, m))
    for i in range(m):
        for j in range(i + 1):
            M[i, j] = np.sum(A[j] * WAW[i])
    asinv = np.array([np.sum(Ai * W) for Ai in A])
    W2 = W @ W
    asinvrd = resi * np.array([np.sum(Ai * W2) for Ai in A]) if resi != 0.0 else np.zeros(m)
    trace = np.trace(W) if resi != 0.0 else 0.0
    return {"M": M, "asinv": asinv, "asinvrd": asinvrd, "tracesinv": trace}


def log_det(S) -> float:
    L = np.linalg.cholesky(S)
    return 2.0 * np.sum(np.log(np.diag(L)))


def max_step(S, dS) -> float:
    """Largest alpha with S + alpha dS psd: 1 / lambda_max(-L^-1 dS L^-T), inf if <= 0."""
    L = np.linalg.cholesky(S)
    Li = np.linalg.inv(L)
    T = -Li @ dS @ Li.T
    lam = np.linalg.eigvalsh(0.5 * (T + T.T))[-1]
    return np.inf if lam <= 0 else 1.0 / lam


def primal_from_dual(C, A, y, dy, mu, perturb=0.0):
    S = dual_slack(C, A, y, 1.0, -1.0, perturb)
    W = np.linalg.inv(S)
    D = sum(d * Ai for d, Ai in zip(dy, A))
    X = mu * (W + W @ D @ W)
    return 0.5 * (X + X.T)


def dimacs(C, A, b, X, S, y):
    """DIMACS errors 1, 2, 5, 6 of (X, y, S) (interface/hdsdp.c:851-866), unscaled data."""
    AX = np.array([np.sum(Ai * X) for Ai in A])
    p = float(np.sum(C * X))
    d = float(b @ y)
    e1 = np.linalg.norm(AX - b) / (1.0 + np.sum(np.abs(b)))
    lmin = np.linalg.eigvalsh(X)[0]
    e2 = max(0.0, -lmin) / (1.0 + np.sum(np.abs(b)))
    e5 = (p - d) / (abs(p) + abs(d) + 1.0)
    e6 = float(np.sum(X * S)) / (abs(p) + abs(d) + 1.0)
    return np.array([e1, e2, e5, e6])
