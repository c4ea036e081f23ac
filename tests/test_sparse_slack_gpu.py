"""The sparse factorisation of the dual slack S on the device (hdsdp_b200/csrc/sparse_chol.cu)
against the dense factorisation and numpy, and solves that use it against the compiled
reference's results and against the dense-factorisation solve."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hdsdp_b200 import _lib, api, instances
from test_solve_gpu import OPTIMAL, check_parity

pytestmark = pytest.mark.gpu


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def laplacian(n, ei, ej, w):
    S = np.zeros((n, n))
    S[ei, ej] = -w
    S[ej, ei] = -w
    S[np.arange(n), np.arange(n)] = -S.sum(axis=1)
    return S


def random_graph(n, m_edges, seed):
    rng = np.random.default_rng(seed)
    e = set()
    while len(e) < m_edges:
        a, b = rng.integers(0, n, 2)
        if a != b:
            e.add((max(a, b), min(a, b)))
    e = np.array(sorted(e), dtype=np.int32)
    return e[:, 0].copy(), e[:, 1].copy(), rng.uniform(0.5, 1.5, len(e))


def sparse_cholesky(S, ei, ej, cap=64, reps=3):
    L = _lib.load()
    n = S.shape[0]
    out = np.zeros(5)
    Sf = np.asfortranarray(S)
    assert L.hdsdpb_sparse_cholesky(n, len(ei), _ip(ei), _ip(ej), _dp(Sf), cap, reps, _dp(out)) == 0
    return out


@pytest.mark.parametrize("n,m_edges", [(300, 900), (3000, 15000)])
def test_sparse_cholesky_logdet_and_definiteness(gpu_lib, n, m_edges):
    ei, ej, w = random_graph(n, m_edges, seed=n)
    S = laplacian(n, ei, ej, w)
    lam = np.linalg.eigvalsh(S)
    Spd = S + 0.5 * np.eye(n)
    out = sparse_cholesky(Spd, ei, ej)
    sign, ref = np.linalg.slogdet(Spd)
    assert out[0] == 1.0 and sign > 0
    assert out[1] == pytest.approx(ref, rel=1e-11)
    assert 0 < out[4] < n
    # a shift that leaves a negative eigenvalue
    out = sparse_cholesky(S - 0.5 * lam[n // 2] * np.eye(n), ei, ej)
    assert out[0] == 0.0


def test_sparse_cholesky_maxcut_n8000(gpu_lib, capsys):
    """The MaxCut workload's slack pattern (n = 8000): same log det as the dense factorisation,
    with the time of both printed."""
    inst = instances.WORKLOADS["maxcut_n8000"]()
    n = inst.n
    C0 = -4.0 * inst.dense(0)  # graph Laplacian
    S = np.asfortranarray(C0 / 4.0 + np.eye(n))
    rows, _ = inst.column(0)
    starts = instances.pack_idx(n, np.arange(n), np.arange(n))
    j = np.searchsorted(starts, rows, side="right") - 1
    i = rows - starts[j] + j
    off = i != j
    ei, ej = i[off].astype(np.int32), j[off].astype(np.int32)
    out = sparse_cholesky(S, ei, ej, reps=5)
    L = _lib.load()
    ld = C.c_double()
    assert L.hdsdpb_cholesky(n, _dp(S), None, C.byref(ld)) == 0
    assert out[0] == 1.0
    assert out[1] == pytest.approx(2.0 * ld.value, rel=1e-11)
    assert out[4] == 4409
    with capsys.disabled():
        print("\nS factorisation, MaxCut n=8000: sparse %.3f ms (front %d), dense %.3f ms" % (out[2], out[4], out[3]))


@pytest.mark.parametrize("name", ["maxcut200", "maxcut60"])
def test_solve_parity_with_sparse_slack(gpu_lib, golden, name):
    """Solves whose PSD checks and log dets all go through the sparse factorisation match
    the compiled reference."""
    from make_golden import SMALL
    inst = SMALL[name]()
    r = api.solve(inst, want_x=False, primal_refinement=False, sparse_slack=1)
    assert r["sparse_slack"]["cones"] == 1 and r["sparse_slack"]["factorisations"] > 0
    check_parity(r, golden["solves"]["%s/psdp0" % name])


def test_solve_maxcut_n2500_sparse_vs_dense(gpu_lib):
    """The trial-point mode picks the sparse factorisation for a sparse MaxCut of order 2500
    and ends where the dense factorisation's solve ends."""
    inst = instances.maxcut(2500, seed=9, n_edges=12500, weights=(0.5, 1.5))
    a = api.solve(inst, want_x=False, primal_refinement=False, sparse_slack=-1)
    b = api.solve(inst, want_x=False, primal_refinement=False, sparse_slack=0)
    assert a["sparse_slack"]["cones"] == 1 and b["sparse_slack"]["cones"] == 0
    assert a["status_after_check"] == b["status_after_check"] == OPTIMAL
    assert abs(a["iters"] - b["iters"]) <= 2
    assert a["dobj"] == pytest.approx(b["dobj"], rel=1e-7)
    assert a["pobj"] == pytest.approx(b["pobj"], rel=1e-7)


def test_multiblock_with_sparse_slack(gpu_lib, golden):
    prob = instances.multiblock_case("mb4_n500")
    r = api.solve_problem(prob, sparse_slack=1)
    check_parity(r, golden["multiblock_solves"]["mb4_n500"])


def test_sparse_congruence(gpu_lib):
    """The Lanczos operator on the sparse factor: with D = S it is the identity, t = L^-T x
    satisfies t^T S t = x^T x, and with D = -dS its spectrum is that of the pencil
    (-dS, S), the same as through the dense factor."""
    L = _lib.load()
    rng = np.random.default_rng(2)
    for n, m_edges in ((600, 2400), (200, 600)):
        ei, ej, w = random_graph(n, m_edges, seed=n)
        S = laplacian(n, ei, ej, w) + 0.7 * np.eye(n)
        Sf = np.asfortranarray(S)
        x = rng.standard_normal(n)
        y, t = np.zeros(n), np.zeros(n)
        assert L.hdsdpb_sparse_congruence(n, len(ei), _ip(ei), _ip(ej), _dp(Sf), _dp(Sf), _dp(x), _dp(y), _dp(t)) == 0
        np.testing.assert_allclose(y, x, rtol=0, atol=1e-11 * np.abs(x).max())
        assert t @ S @ t == pytest.approx(x @ x, rel=1e-12)
    # n = 200: the whole operator for D = -dS, against Lc^-1 (-dS) Lc^-T of the dense factor
    dS = laplacian(n, ei, ej, rng.uniform(-1, 1, len(ei))) + np.diag(rng.uniform(-1, 1, n))
    D = np.asfortranarray(-dS)
    T = np.zeros((n, n))
    e = np.zeros(n)
    for k in range(n):
        e[:] = 0.0
        e[k] = 1.0
        assert L.hdsdpb_sparse_congruence(n, len(ei), _ip(ei), _ip(ej), _dp(Sf), _dp(D), _dp(e), _dp(y), None) == 0
        T[:, k] = y
    Lc = np.linalg.cholesky(S)
    Tref = np.linalg.solve(Lc, np.linalg.solve(Lc, D).T).T
    np.testing.assert_allclose(T, T.T, atol=1e-10 * np.abs(T).max())
    np.testing.assert_allclose(np.linalg.eigvalsh(0.5 * (T + T.T)), np.linalg.eigvalsh(0.5 * (Tref + Tref.T)),
                               atol=1e-10 * np.abs(Tref).max())


@pytest.mark.parametrize("kind", ["tree", "dense"])
def test_sparse_cholesky_edge_patterns(gpu_lib, kind):
    """A tree pattern is eliminated completely (no dense front); a dense pattern (degrees
    above the cap) eliminates nothing and the front is the whole matrix."""
    n = 300
    if kind == "tree":
        rng = np.random.default_rng(4)
        ei = np.arange(1, n, dtype=np.int32)
        ej = np.array([rng.integers(0, i) for i in range(1, n)], dtype=np.int32)
    else:
        ei, ej, _ = random_graph(n, n * 80, seed=9)
    w = np.random.default_rng(5).uniform(0.5, 1.5, len(ei))
    S = laplacian(n, ei, ej, w) + 0.3 * np.eye(n)
    out = sparse_cholesky(S, ei, ej, reps=2)
    sign, ref = np.linalg.slogdet(S)
    assert out[0] == 1.0 and sign > 0
    assert out[1] == pytest.approx(ref, rel=1e-11)
    assert out[4] == (0 if kind == "tree" else n)
    L = _lib.load()
    x = np.random.default_rng(6).standard_normal(n)
    y, t = np.zeros(n), np.zeros(n)
    Sf = np.asfortranarray(S)
    assert L.hdsdpb_sparse_congruence(n, len(ei), _ip(ei), _ip(ej), _dp(Sf), _dp(Sf), _dp(x), _dp(y), _dp(t)) == 0
    np.testing.assert_allclose(y, x, rtol=0, atol=1e-10 * np.abs(x).max())
    assert t @ S @ t == pytest.approx(x @ x, rel=1e-11)
