"""The symmetric indefinite factorisation of the Schur complement (LDL^T with Bunch-Kaufman
pivoting, the solver the reference switches M to when its Cholesky fails,
linalg/hdsdp_linsolver.c:1118-1190 and :1367-1380): the kernels through the C-ABI against
NumPy, and whole solves that factor every M this way against the compiled reference."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hdsdp_b200 import api, instances
from make_golden import FULL, SMALL
from oracle import ldl_ref as R
from test_solve_gpu import check_parity

pytestmark = pytest.mark.gpu

_dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))


def ldl_solve(L, S, b):
    S = np.asfortranarray(S, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    out = np.zeros(3, dtype=np.int32)
    r = L.hdsdpb_ldl_solve(S.shape[0], _dp(S), _dp(b), _dp(x), out.ctypes.data_as(C.POINTER(C.c_int)))
    return r, x, out


def _matrices(n, rng):
    B = rng.standard_normal((n, n))
    yield "random", (B + B.T) / 2
    Z = rng.standard_normal((n, n))
    Z = (Z + Z.T) / 2
    np.fill_diagonal(Z, 0.0)               # every pivot search goes to the row test
    yield "zero_diagonal", Z
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = rng.uniform(0.5, 2.0, n) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    yield "known_spectrum", (Q * ev) @ Q.T
    P = rng.standard_normal((n, n))
    yield "positive_definite", P @ P.T + n * np.eye(n)


# orders on the one-block path (<= 384) and on the cooperative grid
@pytest.mark.parametrize("n", [1, 2, 7, 33, 200, 384, 385, 700, 1500])
def test_ldl_solve_against_numpy(gpu_lib, n):
    rng = np.random.default_rng(100 + n)
    for kind, S in _matrices(n, rng):
        if kind == "zero_diagonal" and n == 1:
            continue   # the zero matrix
        b = rng.standard_normal(n)
        r, x, out = ldl_solve(gpu_lib, S, b)
        assert r == 0, (kind, r)
        ev = np.linalg.eigvalsh(S)
        # the inertia of D is the inertia of S (Sylvester's law); 2 x 2 blocks are indefinite
        assert out[1] == int((ev < 0).sum()) and out[2] == int((ev > 0).sum()), (kind, out)
        if kind == "positive_definite":
            assert out[0] == 0
        if kind == "zero_diagonal" and n >= 2:
            assert out[0] >= 1
        # backward error of a stable solve
        res = np.linalg.norm(S @ x - b) / (np.linalg.norm(S, 1) * np.linalg.norm(x) + np.linalg.norm(b))
        assert res < 1e-14 * max(1.0, np.sqrt(n)), (kind, res)
        xr = np.linalg.solve(S, b)
        cond = np.linalg.cond(S)
        assert np.linalg.norm(x - xr) <= 1e-13 * cond * np.linalg.norm(xr) + 1e-300, kind


# one-block and cooperative-grid orders
@pytest.mark.parametrize("n", [40, 200, 385, 700])
def test_ldl_pivots_match_lapack_restatement(gpu_lib, n):
    """The device factorisation takes the pivots of the restatement of LAPACK's Bunch-Kaufman
    (oracle/ldl_ref.py, itself checked against scipy.linalg.ldl): the same number of 2 x 2
    blocks and the same inertia, and the same solution."""
    rng = np.random.default_rng(500 + n)
    for kind in ("random", "zero_diagonal", "small_diagonal"):
        B = rng.standard_normal((n, n))
        S = (B + B.T) / 2
        if kind == "zero_diagonal":
            np.fill_diagonal(S, 0.0)
        elif kind == "small_diagonal":
            S[np.diag_indices(n)] *= 0.1
        b = rng.standard_normal(n)
        F = R.bunch_kaufman(S)
        r, x, out = ldl_solve(gpu_lib, S, b)
        assert r == 0, kind
        assert tuple(out) == R.inertia(F), kind
        xr = R.solve(F, b)
        cond = np.linalg.cond(S)
        assert np.linalg.norm(x - xr) <= 1e-13 * cond * np.linalg.norm(xr), kind


def test_ldl_edge_cases(gpu_lib):
    L = gpu_lib
    # order 0, a 2 x 2 pivot on its own, singular matrices
    assert ldl_solve(L, np.zeros((0, 0)), np.zeros(0))[0] == 0
    r, x, out = ldl_solve(L, np.array([[0.0, 2.0], [2.0, 0.0]]), np.array([2.0, 4.0]))
    assert r == 0 and list(out) == [1, 1, 1]
    np.testing.assert_allclose(x, [2.0, 1.0], rtol=1e-15)
    assert ldl_solve(L, np.zeros((5, 5)), np.ones(5))[0] == 1
    S = np.diag([1.0, 2.0, 0.0, 3.0])
    assert ldl_solve(L, S, np.ones(4))[0] > 0
    # only the lower triangle is read
    rng = np.random.default_rng(7)
    B = rng.standard_normal((50, 50))
    S = (B + B.T) / 2
    b = rng.standard_normal(50)
    r1, x1, _ = ldl_solve(L, S, b)
    r2, x2, _ = ldl_solve(L, np.tril(S) + np.triu(np.full((50, 50), 1e30), 1), b)
    assert r1 == r2 == 0
    np.testing.assert_array_equal(x1, x2)
    # a NaN pivot is reported, not propagated into a result
    S[0, 0] = np.nan
    assert ldl_solve(L, S, b)[0] == 1


@pytest.mark.parametrize("name", ["maxcut60", "maxcut200", "theta40", "rank1_50_80"])
def test_solve_with_ldl_schur(gpu_lib, name, golden):
    """Every factorisation of M through LDL^T: the same path as the reference's."""
    inst = SMALL[name]()
    r = api.solve(inst, want_x=False, primal_refinement=False, schur_ldl=1)
    check_parity(r, golden["solves"]["%s/psdp0" % name])
    base = api.solve(inst, want_x=False, primal_refinement=False)
    assert r["iters"] == base["iters"]
    assert r["dobj"] == pytest.approx(base["dobj"], rel=1e-9, abs=1e-10)


def test_full_size_solve_with_ldl_schur(gpu_lib, golden):
    """The rank-one workload (m = 2000): LDL^T on the cooperative grid at every iteration."""
    inst = FULL["rank1_n1000_m2000"]()
    r = api.solve(inst, want_x=False, primal_refinement=False, schur_ldl=1)
    check_parity(r, golden["solves"]["rank1_n1000_m2000/psdp0"])


def test_multiblock_solve_with_ldl_schur(gpu_lib, golden):
    for name in ("mb3", "mb2_lp", "mb6_sparse"):
        prob = instances.multiblock_case(name)
        r = api.solve_problem(prob, schur_ldl=1)
        assert not r["sparse_schur"]["arrow"]
        check_parity(r, golden["multiblock_solves"][name])
