"""GPU kernels through the C-ABI against the reference's golden vectors, the
NumPy restatement and NumPy linear algebra (FP64 throughout)."""
from __future__ import annotations

import numpy as np
import pytest

from hdsdp_b200 import api, instances
from make_golden import SMALL, probe_point
from oracle import kernels_ref as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(SMALL))
def test_schur_matches_reference(gpu_lib, name, golden, golden_arrays):
    inst = SMALL[name]()
    y, resi, _ = probe_point(inst)
    r = api.schur_probe(inst, y, resi)
    M = golden_arrays["M/" + name]
    assert np.abs(r["M"] - M).max() <= 1e-11 * np.abs(M).max()
    for key in ("asinv", "asinvrd"):
        g = golden_arrays[key + "/" + name]
        assert np.abs(r[key] - g).max() <= 1e-11 * max(1.0, np.abs(g).max())
    assert r["tracesinv"] == pytest.approx(golden["probes"][name]["tracesinv"], rel=1e-11)


@pytest.mark.parametrize("name", sorted(SMALL))
def test_ratio_test_matches_reference(gpu_lib, name, golden):
    inst = SMALL[name]()
    y, resi, dy = probe_point(inst)
    step, logdet = api.ratio_probe(inst, y, resi, dy, 0.5)
    p = golden["probes"][name]
    # same Lanczos start vector, subspace size and stopping rule as the reference
    assert step == pytest.approx(p["step"], rel=1e-8)
    assert logdet == pytest.approx(p["logdet"], rel=1e-12, abs=1e-9)


def test_schur_rank_one_full_size(gpu_lib):
    """Rank-one workload n=1000, m=2000: M_ij = s_i s_j (a_i^T W a_j)^2 (dense rank-one GEMM path)."""
    inst = instances.WORKLOADS["rank1_n1000_m2000"]()
    n, m = inst.n, inst.m
    rng = np.random.default_rng(7)
    y = -np.abs(rng.standard_normal(m)) * 1e-3
    resi = -2.0
    C = K.unpack_column(n, *inst.column(0))
    A1 = np.stack([K.rank_one_factor(n, *inst.column(k + 1)) for k in range(m)], axis=1)
    S = C - (A1 * y) @ A1.T - resi * np.eye(n)
    W = np.linalg.inv(S)
    G = A1.T @ W @ A1
    Mref = np.tril(G * G)
    r = api.schur_probe(inst, y, resi)
    assert np.abs(r["M"] - Mref).max() <= 1e-10 * np.abs(Mref).max()
    np.testing.assert_allclose(r["asinv"], np.diag(G), rtol=1e-10)
    np.testing.assert_allclose(r["asinvrd"], resi * np.einsum("ik,ik->k", W @ A1, W @ A1), rtol=1e-10)


def _spd(n, seed, cond=1e3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.logspace(0, np.log10(cond), n)
    return (Q * ev) @ Q.T


# up to 2100 the one-launch kernel; 8300 the recursive form without K
@pytest.mark.parametrize("n", [1, 2, 31, 64, 65, 127, 200, 513, 1000, 2100, 8300])
def test_cholesky_and_inverse(gpu_lib, n):
    S = _spd(n, n)
    L, logdiag, pd = api.cholesky(S)
    assert pd
    Lref = np.linalg.cholesky(S)
    assert np.abs(L - Lref).max() <= 1e-11 * np.abs(Lref).max()
    assert logdiag == pytest.approx(np.log(np.diag(Lref)).sum(), rel=1e-12, abs=1e-12)
    Si = api.inverse(S)
    assert np.abs(Si @ S - np.eye(n)).max() <= 1e-9


# the one-launch kernel with K (up to 3840), just above the crossover to the recursive form
# (one split), and an order whose halves split again
@pytest.mark.parametrize("n", [700, 2100, 3840, 3904, 4577, 5999])
def test_cholesky_with_inverse_factor(gpu_lib, n):
    import ctypes as C
    S = np.asfortranarray(_spd(n, 3 * n))
    L = np.zeros((n, n), order="F")
    K = np.zeros((n, n), order="F")
    dp = C.POINTER(C.c_double)
    r = gpu_lib.hdsdpb_cholesky_inverse_factor(n, S.ctypes.data_as(dp), L.ctypes.data_as(dp), K.ctypes.data_as(dp))
    assert r == 0
    Lref = np.linalg.cholesky(S)
    assert np.abs(L - Lref).max() <= 1e-11 * np.abs(Lref).max()
    assert np.abs(np.triu(K, 1)).max() == 0.0
    assert np.abs(K @ Lref - np.eye(n)).max() <= 1e-10


@pytest.mark.parametrize("n", [5, 64, 300])
def test_cholesky_detects_indefinite(gpu_lib, n):
    S = _spd(n, 3)
    S[n // 2, n // 2] = -1.0
    _, _, pd = api.cholesky(S)
    assert not pd
    assert api.inverse(S) is None


def test_empty_factorisation(gpu_lib):
    L, logdiag, pd = api.cholesky(np.zeros((0, 0)))
    assert pd and logdiag == 0.0 and L.shape == (0, 0)


@pytest.mark.parametrize("M,N,Kd", [(1, 1, 1), (65, 33, 17), (300, 200, 150), (1000, 1000, 2000),
                                    (1500, 1400, 64), (70, 50, 0)])
@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True), (True, True)])
def test_gemm(gpu_lib, M, N, Kd, tA, tB):
    rng = np.random.default_rng(M * 7 + N + Kd)
    A = rng.standard_normal((Kd, M) if tA else (M, Kd))
    B = rng.standard_normal((N, Kd) if tB else (Kd, N))
    C0 = rng.standard_normal((M, N))
    out = api.gemm(0.7, A, B, beta=-0.3, Cm=C0, transA=tA, transB=tB)
    ref = 0.7 * ((A.T if tA else A) @ (B.T if tB else B)) - 0.3 * C0
    assert np.abs(out - ref).max() <= 1e-12 * max(1.0, Kd) * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 200, 1000, 2100, 9600])
def test_cholesky_solve(gpu_lib, n):
    """Blocked forward / backward substitution with the factor (the Schur-solve path for
    m >= 6000); n = 9600 gives 150 row blocks, so some CTAs own two."""
    rng = np.random.default_rng(n + 11)
    if n <= 2100:
        S = _spd(n, n + 1)
    else:
        R = rng.standard_normal((n, 40))
        S = R @ R.T / 40.0 + np.eye(n)
    b = rng.standard_normal(n)
    x = api.cholesky_solve(S, b)
    assert x is not None
    res = np.abs(S @ x - b).max()
    assert res <= 1e-11 * np.abs(S).max() * max(1.0, np.abs(x).max())
    x2 = api.cholesky_solve(S, b)  # a second solve reuses nothing stale
    np.testing.assert_array_equal(x2, x)


def test_cholesky_solve_indefinite(gpu_lib):
    S = _spd(100, 5)
    S[50, 50] = -1.0
    assert api.cholesky_solve(S, np.ones(100)) is None


@pytest.mark.parametrize("n", [1, 37, 64, 65, 100, 128, 200, 333, 512, 1000])
def test_cholesky_batch_matches_whole_gpu_kernel(gpu_lib, n):
    """The one-CTA-per-matrix factorisation of the multi-cone path (mode 0) gives the
    cooperative whole-GPU kernel's L, K = L^-1, log det and status to the bit (mode 1), and
    matches NumPy; the third matrix is indefinite."""
    import ctypes as C
    from hdsdp_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(n)
    mats = []
    for q in range(3):
        G = rng.standard_normal((n, n))
        S = G @ G.T / n + np.eye(n)
        if q == 2:
            S[n // 2, n // 2] = -1.0 - np.abs(S[n // 2]).sum()
        mats.append(S)
    Sall = np.ascontiguousarray(np.stack([np.asfortranarray(S).ravel(order="F") for S in mats]))
    out = {}
    dp = C.POINTER(C.c_double)
    for mode in (0, 1):
        Lo, Ko = np.zeros((3, n * n)), np.zeros((3, n * n))
        ld, st = np.zeros(3), np.zeros(3, dtype=np.int32)
        r = L.hdsdpb_cholesky_batch(3, n, mode, Sall.ctypes.data_as(dp), Lo.ctypes.data_as(dp),
                                    Ko.ctypes.data_as(dp), ld.ctypes.data_as(dp),
                                    st.ctypes.data_as(C.POINTER(C.c_int)))
        assert r == 0
        out[mode] = (Lo, Ko, ld, st)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    Lo, Ko, ld, st = out[0]
    assert list(st) == [0, 0, 1]
    for q in range(2):
        Lq = Lo[q].reshape(n, n, order="F")
        Kq = Ko[q].reshape(n, n, order="F")
        Lr = np.linalg.cholesky(mats[q])
        assert np.abs(Lq - Lr).max() <= 1e-12 * max(1.0, np.abs(Lr).max())
        assert np.abs(Kq @ Lq - np.eye(n)).max() <= 1e-10
        assert ld[q] == pytest.approx(np.log(np.diag(Lr)).sum(), rel=1e-12, abs=1e-12)
