"""BF16x3 split-precision products on the tcgen05 tensor cores against FP64 NumPy.

Each FP64 entry is carried as hi + lo BF16 parts (representation error
2^-18 |x|) and the product keeps hi*hi + hi*lo + lo*hi with FP32
accumulation, so every entry is within about 3 * 2^-18 of sum_k |a_k b_k|
plus the FP32 accumulation error; the tolerance below is 6e-5 of that sum.
"""
from __future__ import annotations

import numpy as np
import pytest

from hdsdp_b200 import api
from oracle import kernels_ref as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (128, 128, 64), (300, 200, 150), (129, 257, 65),
                                   (1000, 2000, 1000), (2000, 2000, 1000), (3000, 2500, 700)])
@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True)])
def test_split_gemm_accuracy(gpu_lib, M, N, K, tA, tB):
    rng = np.random.default_rng(M + 3 * N + 7 * K)
    A = rng.standard_normal((K, M) if tA else (M, K))
    B = rng.standard_normal((N, K) if tB else (K, N))
    opA = A.T if tA else A
    opB = B.T if tB else B
    out = api.split_gemm(A, B, transA=tA, transB=tB)
    ref = opA @ opB
    bound = np.abs(opA) @ np.abs(opB)
    assert np.all(np.abs(out - ref) <= 6e-5 * bound + 1e-300)
    # the split keeps far more than BF16 alone (2^-9 per entry)
    assert np.abs(out - ref).max() <= 2e-4 * bound.max()


def test_split_gemm_wide_dynamic_range(gpu_lib):
    rng = np.random.default_rng(5)
    A = rng.standard_normal((256, 192)) * np.exp(rng.uniform(-20, 20, size=(256, 192)))
    B = rng.standard_normal((192, 160))
    out = api.split_gemm(A, B)
    ref = A @ B
    bound = np.abs(A) @ np.abs(B)
    assert np.all(np.abs(out - ref) <= 6e-5 * bound)


def test_split_schur_rank_one(gpu_lib):
    """Rank-one Schur block in split precision (B = L^-1 A1, G = B^T B) against the FP64 build."""
    from hdsdp_b200 import instances
    inst = instances.WORKLOADS["rank1_n1000_m2000"]()
    rng = np.random.default_rng(7)
    y = -np.abs(rng.standard_normal(inst.m)) * 1e-3
    resi = -2.0
    ref = api.schur_probe(inst, y, resi, precision=0)
    spl = api.schur_probe(inst, y, resi, precision=1)
    scale = np.abs(ref["M"]).max()
    assert np.abs(spl["M"] - ref["M"]).max() <= 1e-4 * scale
    np.testing.assert_allclose(spl["asinv"], ref["asinv"], rtol=1e-4)
    np.testing.assert_allclose(spl["asinvrd"], ref["asinvrd"], rtol=1e-4)


def _maxcut_probe(n):
    from hdsdp_b200 import instances
    inst = instances.maxcut(n, 10.0 / n, seed=11)
    rows, vals = inst.column(0)
    i, j = K.packed_to_ij(n, rows)
    deg = -4.0 * np.asarray(vals)[i == j]          # C = -L/4: the diagonal holds -degree/4
    y = -(0.5 * deg.max() + 1.0) * np.ones(inst.m)  # S = C - diag(y) + 2 I is safely positive definite
    return inst, y, -2.0


def test_split_inverse_maxcut_schur(gpu_lib):
    """S^-1 = K^T K formed in split precision (n >= 1024) for the sparse rank-one block
    of a MaxCut instance, M_ij = (S^-1)_ij^2, against the FP64 build: each entry of
    S^-1 is within about 6e-5 sqrt(W_ii W_jj) (Cauchy-Schwarz on the BF16x3 bound)."""
    inst, y, resi = _maxcut_probe(1100)
    ref = api.schur_probe(inst, y, resi, precision=0)
    spl = api.schur_probe(inst, y, resi, precision=1)
    d = np.sqrt(np.diag(ref["M"]))
    bound = 2e-4 * np.tril(np.outer(d, d))
    assert np.all(np.abs(spl["M"] - ref["M"]) <= bound + 1e-300)
    np.testing.assert_allclose(spl["asinv"], ref["asinv"], rtol=1e-4)
    np.testing.assert_allclose(spl["asinvrd"], ref["asinvrd"], rtol=2e-4)
    assert spl["tracesinv"] == pytest.approx(ref["tracesinv"], rel=1e-4)


@pytest.mark.parametrize("mode", [1, 2])
def test_split_solve_maxcut(gpu_lib, mode):
    """MaxCut n = 1100 solved with split-precision Schur assembly (1: every build,
    2: until the gap reaches 1e-3, the mode meant for use) against the FP64 GPU solve."""
    from hdsdp_b200 import instances
    inst = instances.maxcut(1100, 10.0 / 1100, seed=11)
    ref = api.solve(inst, want_x=False, primal_refinement=False, precision=0)
    spl = api.solve(inst, want_x=False, primal_refinement=False, precision=mode)
    print("mode %d: iters %d vs %d, dobj %.12g vs %.12g, pobj %.12g vs %.12g, errs %s"
          % (mode, spl["iters"], ref["iters"], spl["dobj"], ref["dobj"], spl["pobj"], ref["pobj"], spl["errs"]))
    assert ref["status_after_check"] == 3 and spl["status_after_check"] == 3
    assert spl["dobj"] == pytest.approx(ref["dobj"], rel=1e-6)
    if mode == 2:
        # the last iterations run in FP64, as in the reference: full parity
        assert spl["pobj"] == pytest.approx(ref["pobj"], rel=1e-6)
        assert max(spl["errs"][0], spl["errs"][1]) <= 1e-7
        assert abs(spl["iters"] - ref["iters"]) <= 2
    else:
        # split builds throughout: the inexact Newton directions take their own path,
        # and X is recovered from a split-precision Newton system (about 1e-4 relative)
        assert spl["pobj"] == pytest.approx(ref["pobj"], rel=1e-3)
