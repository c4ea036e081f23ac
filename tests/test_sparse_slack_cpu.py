"""Ordering of the sparse factorisation of the dual slack S (multiple-minimum-degree rounds
and a dense front, hdsdp_b200/csrc/sparse_chol.cu), host side only.

The library's ordering (hdsdpb_sparse_analyse, no device work) is checked against a
Python restatement of the same rules, and the numerical scheme built on it (scale the
round's independent columns, apply their Schur updates, factor the dense front) is run in
numpy and checked against numpy's log det and definiteness. The device kernels are
checked against the dense factorisation in tests/test_sparse_slack_gpu.py.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hdsdp_b200 import _lib, instances
from hdsdp_b200.build import build


def mmd_rounds(n, adj, cap):
    """Rounds of (vertex, sorted neighbours) eliminated and the front: each round takes, in
    (degree, index) order, an independent set of vertices of degree at most
    min(cap, d_min + max(1, d_min // 4)); rounds stop when d_min exceeds cap."""
    A = [set(a) for a in adj]
    alive = [True] * n
    rounds = []
    while True:
        order = sorted((len(A[v]), v) for v in range(n) if alive[v])
        if not order or order[0][0] > cap:
            break
        mind = order[0][0]
        thr = min(cap, mind + max(1, mind // 4))
        mark = [False] * n
        picked = []
        for d, v in order:
            if d > thr:
                break
            if mark[v]:
                continue
            picked.append(v)
            mark[v] = True
            for u in A[v]:
                mark[u] = True
        cols = []
        for v in picked:
            N = sorted(A[v])
            cols.append((v, N))
            for u in N:
                A[u].discard(v)
                A[u].update(w for w in N if w != u)
            A[v] = set()
            alive[v] = False
        rounds.append(cols)
    return rounds, [v for v in range(n) if alive[v]]


def hybrid_logdet(S, rounds, front):
    """(positive definite, log det) by the rounds and a dense front factorisation."""
    W = S.copy()
    logdet = 0.0
    for cols in rounds:
        lv = []
        for v, N in cols:
            d = W[v, v]
            if not d > 0:
                return False, None
            l = np.sqrt(d)
            logdet += 2.0 * np.log(l)
            lv.append((N, W[N, v] / l))
        for N, x in lv:
            W[np.ix_(N, N)] -= np.outer(x, x)
    if front:
        try:
            Lf = np.linalg.cholesky(W[np.ix_(front, front)])
        except np.linalg.LinAlgError:
            return False, None
        logdet += 2.0 * np.log(np.diag(Lf)).sum()
    return True, logdet


def graph(n, m_edges, seed):
    rng = np.random.default_rng(seed)
    e = set()
    while len(e) < m_edges:
        a, b = rng.integers(0, n, 2)
        if a != b:
            e.add((max(a, b), min(a, b)))
    e = np.array(sorted(e), dtype=np.int32)
    adj = [[] for _ in range(n)]
    for a, b in e:
        adj[a].append(int(b))
        adj[b].append(int(a))
    return e[:, 0].copy(), e[:, 1].copy(), [sorted(x) for x in adj]


def analyse(n, ei, ej, cap):
    build()
    L = _lib.load()
    out = np.zeros(5)
    front = np.zeros(n, dtype=np.int32)
    r = L.hdsdpb_sparse_analyse(n, len(ei), ei.ctypes.data_as(C.POINTER(C.c_int)),
                                ej.ctypes.data_as(C.POINTER(C.c_int)), cap,
                                out.ctypes.data_as(C.POINTER(C.c_double)), front.ctypes.data_as(C.POINTER(C.c_int)))
    assert r == 0
    return out, front[:int(out[1])]


@pytest.mark.parametrize("n,m_edges,cap", [(300, 900, 64), (500, 5000, 16), (200, 199, 64), (64, 2016, 32)])
def test_ordering_matches_restatement(n, m_edges, cap):
    ei, ej, adj = graph(n, m_edges, seed=n + m_edges)
    out, front = analyse(n, ei, ej, cap)
    rounds, pfront = mmd_rounds(n, adj, cap)
    assert int(out[0]) == len(rounds)
    assert int(out[2]) == sum(len(c) for c in rounds)
    np.testing.assert_array_equal(front, pfront)
    # every round is an independent set of the graph it is taken from, and every vertex is
    # eliminated once or in the front
    seen = set(pfront)
    for cols in rounds:
        vs = {v for v, _ in cols}
        for v, N in cols:
            assert not (set(N) & vs)
            assert v not in seen
            seen.add(v)
    assert seen == set(range(n))


def test_ordering_maxcut_n8000():
    """The dual-slack pattern of the MaxCut workload (n = 8000, 40,000 edges): 13 rounds,
    a front of 4,409 (17 % of the dense factorisation's flops)."""
    inst = instances.WORKLOADS["maxcut_n8000"]()
    rows, _ = inst.column(0)
    n = inst.n
    starts = instances.pack_idx(n, np.arange(n), np.arange(n))
    j = np.searchsorted(starts, rows, side="right") - 1
    i = rows - starts[j] + j
    off = i != j
    ei, ej = i[off].astype(np.int32), j[off].astype(np.int32)
    out, front = analyse(n, ei, ej, 64)
    adj = [[] for _ in range(n)]
    for a, b in zip(ei.tolist(), ej.tolist()):
        adj[a].append(b)
        adj[b].append(a)
    rounds, pfront = mmd_rounds(n, adj, 64)
    assert (int(out[0]), int(out[1])) == (len(rounds), len(pfront)) == (13, 4409)
    np.testing.assert_array_equal(front, pfront)


@pytest.mark.parametrize("shift,pd", [(1.0, True), (-0.5, False)])
def test_numeric_scheme(shift, pd):
    """The rounds plus a dense front give the log det and the definiteness of S."""
    n = 300
    ei, ej, adj = graph(n, 900, seed=5)
    rng = np.random.default_rng(1)
    w = rng.uniform(0.5, 1.5, len(ei))
    S = np.zeros((n, n))
    S[ei, ej] = -w
    S[ej, ei] = -w
    S[np.arange(n), np.arange(n)] = -S.sum(axis=1)  # graph Laplacian, psd
    lam = np.linalg.eigvalsh(S)
    S += (shift if pd else -0.5 * lam[-1]) * np.eye(n)
    rounds, front = mmd_rounds(n, adj, 64)
    assert len(rounds) > 0
    ok, logdet = hybrid_logdet(S, rounds, front)
    sign, ref = np.linalg.slogdet(S)
    assert ok == pd == (sign > 0 and np.linalg.eigvalsh(S)[0] > 0)
    if pd:
        assert logdet == pytest.approx(ref, rel=1e-12)


def hybrid_factor(S, rounds, front):
    """The numbers the device factor holds: per eliminated vertex l_vv and its column
    entries (l_av for a in N(v)), and the front's dense Cholesky factor."""
    W = S.copy()
    cols = {}
    for rnd in rounds:
        lv = []
        for v, N in rnd:
            l = np.sqrt(W[v, v])
            x = W[N, v] / l
            cols[v] = (l, N, x)
            lv.append((N, x))
        for N, x in lv:
            W[np.ix_(N, N)] -= np.outer(x, x)
    Lf = np.linalg.cholesky(W[np.ix_(front, front)]) if front else np.zeros((0, 0))
    return cols, Lf


def congruence(D, x, rounds, front, cols, Lf):
    """y = L^-1 D L^-T x in the original order, the way the device applies it: L^-T by the
    front and then the rounds last to first, L^-1 by the rounds first to last and then the
    front."""
    n = len(x)
    t = np.zeros(n)
    if front:
        t[front] = np.linalg.solve(Lf.T, x[front])
    for rnd in reversed(rounds):
        for v, _ in rnd:
            l, N, lv = cols[v]
            t[v] = (x[v] - lv @ t[N]) / l
    w = D @ t
    y = np.zeros(n)
    rem = w.copy()
    for rnd in rounds:
        for v, _ in rnd:
            l, N, lv = cols[v]
            y[v] = rem[v] / l
        for v, _ in rnd:  # the round's columns pushed into the rows below them
            l, N, lv = cols[v]
            rem[N] -= lv * y[v]
    if front:
        y[front] = np.linalg.solve(Lf, rem[front])
    return t, y


@pytest.mark.parametrize("m_edges", [900, 300, 4000])
def test_congruence_scheme(m_edges):
    """With D = S the operator is the identity, and t = L^-T x has t^T S t = x^T x."""
    n = 300
    ei, ej, adj = graph(n, m_edges, seed=m_edges)
    rng = np.random.default_rng(3)
    w = rng.uniform(0.5, 1.5, len(ei))
    S = np.zeros((n, n))
    S[ei, ej] = -w
    S[ej, ei] = -w
    S[np.arange(n), np.arange(n)] = -S.sum(axis=1) + 0.5
    rounds, front = mmd_rounds(n, adj, 64)
    cols, Lf = hybrid_factor(S, rounds, front)
    x = rng.standard_normal(n)
    t, y = congruence(S, x, rounds, front, cols, Lf)
    np.testing.assert_allclose(y, x, atol=1e-10 * np.abs(x).max())
    assert t @ S @ t == pytest.approx(x @ x, rel=1e-11)
