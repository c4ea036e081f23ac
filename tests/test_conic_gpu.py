"""The conic callback interface (include/hdsdp_conic.h) against the compiled reference's.

Both libraries are driven through the same hooks, in the same order, on the same data:
HConeCreate / HConeSetData / HConeProcData / HConePresolveData, then the algorithm hooks
(start, interior checks, log barrier, ratio test, step-and-check, primal and dual
recovery, A X, <C, X>, norms, feature detection) and the KKT manager (HKKTInit,
HKKTBuildUp of each KKT type, HKKTExport, the Schur matrix, HKKTFactorize / HKKTSolve),
as the reference's algorithm calls them (interface/hdsdp_algo.c). Parity: FP64
arithmetic to 1e-11 relative for the Schur quantities, 1e-8 for the Lanczos step bound
and the Schur solve, exact agreement of every yes/no answer.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os

import numpy as np
import pytest

from hdsdp_b200 import _lib, instances
from make_golden import DENSE, SMALL, probe_point
from oracle import ref_api

pytestmark = pytest.mark.gpu

DENSE_SDP, LP, SCALAR_BOUND = 4, 1, 3
VAR, CHECK, STEP = 0, 1, 2
INFEASIBLE, CORRECTOR, HOMOGENEOUS = 0, 1, 2
vp, ip, dp, i, d = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, C.c_double


def _bind_reference():
    L = ref_api.lib()
    sig = {
        "HConeCreate": ([C.POINTER(vp)], i), "HConeSetData": ([vp, vp], i), "HConeProcData": ([vp], i),
        "HConePresolveData": ([vp], i), "HConeDestroy": ([C.POINTER(vp)], None),
        "HConeDetectFeature": ([vp, dp, ip, dp], None), "HConeSetStart": ([vp, d], None),
        "HConeUpdate": ([vp, d, dp], None), "HConeRatioTest": ([vp, d, dp, d, i, dp], i),
        "HConeGetSymNnz": ([vp], C.c_int64), "HConeGetDim": ([vp], i), "HConeGetCoeffNorm": ([vp, i], d),
        "HConeGetObjNorm": ([vp, i], d), "HConeGetLogBarrier": ([vp, d, dp, i, dp], i),
        "HConeAddStepToBufferAndCheck": ([vp, d, i, ip], i), "HConeCheckIsInterior": ([vp, d, dp, ip], i),
        "HConeCheckIsInteriorExpert": ([vp, d, d, dp, d, i, ip], i), "HConeReduceResi": ([vp, d], None),
        "HConeSetPerturb": ([vp, d], None), "HConeGetPrimal": ([vp, d, dp, dp, dp, dp], None),
        "HConeGetDual": ([vp, dp, dp], None), "HConeComputeATimesX": ([vp, dp, dp], None),
        "HConeComputeTraceCX": ([vp, dp], d), "HConeScalByConstant": ([vp, d], None),
        "HKKTCreate": ([C.POINTER(vp)], i), "HKKTInit": ([vp, i, i, C.POINTER(vp)], i),
        "HKKTBuildUp": ([vp, i], i), "HKKTBuildUpExtraCone": ([vp, vp, i], i),
        "HKKTExport": ([vp, dp, dp, dp, dp, dp, dp, dp], None), "HKKTFactorize": ([vp], i),
        "HKKTSolve": ([vp, dp, dp], i), "HKKTDestroy": ([C.POINTER(vp)], None),
        "oracle_kkt_matrix": ([vp, i, dp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


@contextlib.contextmanager
def _quiet():
    """The reference prints from its KKT set-up; keep the test output clean."""
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    os.close(devnull)
    try:
        yield
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def _p(a):
    return a.ctypes.data_as(dp)


class Side:
    """One library's cones and KKT object over the same user data."""

    def __init__(self, L, blocks, m):
        self.L, self.m, self.keep, self.uds, self.cones = L, m, [], [], []
        for kind, dim, Ap, Ai, Ax in blocks:
            arrs = [np.ascontiguousarray(Ap, np.int32), np.ascontiguousarray(Ai, np.int32),
                    np.ascontiguousarray(Ax, np.float64)]
            self.keep.append(arrs)
            ud = vp()
            assert L.HUserDataCreate(C.byref(ud)) == 0
            L.HUserDataSetConeData(ud, kind, m, dim, arrs[0].ctypes.data_as(ip), arrs[1].ctypes.data_as(ip),
                                   _p(arrs[2]))
            self.uds.append(ud)
            c = vp()
            assert L.HConeCreate(C.byref(c)) == 0
            assert L.HConeSetData(c, ud) == 0
            assert L.HConeProcData(c) == 0
            assert L.HConePresolveData(c) == 0
            self.cones.append(c)
        self.kkt = vp()

    def init_kkt(self, n_cones):
        assert self.L.HKKTCreate(C.byref(self.kkt)) == 0
        arr = (vp * n_cones)(*[c.value for c in self.cones[:n_cones]])
        self._arr = arr
        with _quiet():
            assert self.L.HKKTInit(self.kkt, self.m, n_cones, arr) == 0

    def export(self):
        a, ard, acs = np.zeros(self.m), np.zeros(self.m), np.zeros(self.m)
        sc = [C.c_double() for _ in range(4)]
        self.L.HKKTExport(self.kkt, _p(a), _p(ard), _p(acs), C.byref(sc[0]), C.byref(sc[1]), C.byref(sc[2]),
                          C.byref(sc[3]))
        return a, ard, acs, [x.value for x in sc]

    def close(self):
        if self.kkt.value:
            self.L.HKKTDestroy(C.byref(self.kkt))
        for c in self.cones:
            self.L.HConeDestroy(C.byref(c))
        for ud in self.uds:
            self.L.HUserDataDestroy(C.byref(ud))


def _close(a, b, rel, what):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = max(1.0, float(np.abs(b).max()) if b.size else 1.0)
    assert float(np.abs(a - b).max() if a.size else 0.0) <= rel * scale, (what, a, b)


def _interior_point(inst, y):
    """A dual point near y with C - A^T y positive definite (no residual term)."""
    from oracle import kernels_ref as K
    Cm, A = K.dense_data(inst)
    n = inst.n
    cands = [np.zeros_like(y), 1e-3 * y, y - (n + 10.0)]
    if np.allclose(A[0], np.eye(n)):
        t = y.copy()
        t[0] -= n + 10.0
        cands.insert(0, t)
    for c in cands:
        if np.linalg.eigvalsh(K.dual_slack(Cm, A, c))[0] > 1e-3:
            return np.ascontiguousarray(c)
    raise AssertionError("no interior point found")


def _both(blocks, m):
    R = _bind_reference()
    G = _lib.load()
    with _quiet():
        return Side(G, blocks, m), Side(R, blocks, m)


CASES = {k: SMALL[k] for k in ("theta40", "rank1_50_80", "maxcut60")}
CASES.update({"dense40": DENSE["dense40"]})


@pytest.mark.parametrize("name", sorted(CASES))
def test_sdp_cone_hooks_match_reference(gpu_lib, name):
    inst = CASES[name]()
    m, n = inst.m, inst.n
    g, r = _both([(DENSE_SDP, n, inst.Ap, inst.Ai, inst.Ax)], m)
    try:
        gc, rc = g.cones[0], r.cones[0]
        assert g.L.HConeGetDim(gc) == r.L.HConeGetDim(rc) == n
        for which in (1, 2):
            _close(g.L.HConeGetCoeffNorm(gc, which), r.L.HConeGetCoeffNorm(rc, which), 1e-12, "coeff norm")
            _close(g.L.HConeGetObjNorm(gc, which), r.L.HConeGetObjNorm(rc, which), 1e-12, "obj norm")
        fi_g, fi_r = np.zeros(20, np.int32), np.zeros(20, np.int32)
        fd_g, fd_r = np.zeros(20), np.zeros(20)
        b = np.ascontiguousarray(inst.b)
        g.L.HConeDetectFeature(gc, _p(b), fi_g.ctypes.data_as(ip), _p(fd_g))
        r.L.HConeDetectFeature(rc, _p(b), fi_r.ctypes.data_as(ip), _p(fd_r))
        np.testing.assert_array_equal(fi_g, fi_r)
        _close(fd_g, fd_r, 1e-12, "features")

        y, resi, dy = probe_point(inst)
        out = {}
        for side, c in (("g", g), ("r", r)):
            L, cone = c.L, c.cones[0]
            L.HConeSetStart(cone, resi)
            inn = C.c_int()
            assert L.HConeCheckIsInterior(cone, 1.0, _p(y), C.byref(inn)) == 0
            ld = C.c_double()
            assert L.HConeGetLogBarrier(cone, 0.0, None, VAR, C.byref(ld)) == 0
            st = C.c_double()
            with _quiet():
                assert L.HConeRatioTest(cone, 0.0, _p(dy), 0.5, VAR, C.byref(st)) == 0
            half, inn2, ld2 = 0.5 * st.value, C.c_int(), C.c_double()
            assert L.HConeAddStepToBufferAndCheck(cone, half, CHECK, C.byref(inn2)) == 0
            assert L.HConeGetLogBarrier(cone, 0.0, None, CHECK, C.byref(ld2)) == 0
            # a point beyond the step bound is not interior
            inn3 = C.c_int()
            assert L.HConeAddStepToBufferAndCheck(cone, 1.5 * st.value, CHECK, C.byref(inn3)) == 0
            inn4 = C.c_int()
            y2 = np.ascontiguousarray(y + 0.25 * st.value * dy)
            assert L.HConeCheckIsInteriorExpert(cone, 1.0, -1.0, _p(y2), -resi, CHECK, C.byref(inn4)) == 0
            out[side] = (inn.value, ld.value, st.value, inn2.value, ld2.value, inn3.value, inn4.value)
        (gi, gld, gst, gi2, gld2, gi3, gi4), (ri, rld, rst, ri2, rld2, ri3, ri4) = out["g"], out["r"]
        assert (gi, gi2, gi4) == (ri, ri2, ri4) == (1, 1, 1)
        assert gi3 == ri3
        _close(gld, rld, 1e-12, "log det")
        _close(gst, rst, 1e-8, "step bound")
        _close(gld2, rld2, 1e-10, "log det after the step")

        # the KKT manager: every build type at the same point
        g.init_kkt(1)
        r.init_kkt(1)
        for side in (g, r):
            side.L.HConeSetStart(side.cones[0], resi)
            side.L.HConeUpdate(side.cones[0], 1.0, _p(y))
        for typ in (INFEASIBLE, CORRECTOR, HOMOGENEOUS):
            with _quiet():
                assert g.L.HKKTBuildUp(g.kkt, typ) == 0
                assert r.L.HKKTBuildUp(r.kkt, typ) == 0
            ga, gard, gacs, gsc = g.export()
            ra, rard, racs, rsc = r.export()
            _close(ga, ra, 1e-11, "ASinv %d" % typ)
            _close(gard, rard, 1e-11, "ASinvRdSinv %d" % typ)
            if typ == HOMOGENEOUS:
                _close(gacs, racs, 1e-10, "ASinvCSinv")
                _close(gsc[:3], rsc[:3], 1e-10, "C scalars")
            if typ != CORRECTOR:
                _close(gsc[3], rsc[3], 1e-11, "trace S^-1")
                Mg, Mr = np.zeros((m, m), order="F"), np.zeros((m, m), order="F")
                assert g.L.HKKTGetMatrix(g.kkt, _p(Mg)) == 0
                assert r.L.oracle_kkt_matrix(r.kkt, m, _p(Mr)) == 0
                _close(np.tril(Mg), np.tril(Mr), 1e-11, "M %d" % typ)
        # factor and solve M x = ASinv (the reference iterates CG to 1e-12 or factors)
        with _quiet():
            assert g.L.HKKTBuildUp(g.kkt, INFEASIBLE) == 0
            assert r.L.HKKTBuildUp(r.kkt, INFEASIBLE) == 0
            assert g.L.HKKTFactorize(g.kkt) == 0
            assert r.L.HKKTFactorize(r.kkt) == 0
        rhs = np.ascontiguousarray(g.export()[0])
        xg, xr = np.zeros(m), np.zeros(m)
        with _quiet():
            assert g.L.HKKTSolve(g.kkt, _p(rhs.copy()), _p(xg)) == 0
            assert r.L.HKKTSolve(r.kkt, _p(rhs.copy()), _p(xr)) == 0
        _close(xg, xr, 1e-8, "Schur solve")

        # primal and dual recovery, A X, <C, X> at a point where S = C - A^T y is interior
        yv = _interior_point(inst, y)
        mu = 0.1
        Xg, Xr = np.zeros((n, n), order="F"), np.zeros((n, n), order="F")
        Sg, Sr = np.zeros((n, n), order="F"), np.zeros((n, n), order="F")
        aux = np.zeros((n, n), order="F")
        dyv = np.ascontiguousarray(0.01 * dy)
        g.L.HConeGetPrimal(g.cones[0], mu, _p(yv), _p(dyv), _p(Xg), _p(aux))
        r.L.HConeGetPrimal(r.cones[0], mu, _p(yv), _p(dyv), _p(Xr), _p(aux))
        _close(Xg, Xr, 1e-10, "X")
        g.L.HConeGetDual(g.cones[0], _p(Sg), None)
        r.L.HConeGetDual(r.cones[0], _p(Sr), None)
        _close(Sg, Sr, 1e-12, "S")
        axg, axr = np.zeros(m), np.zeros(m)
        Xs = np.asfortranarray(Xr)
        g.L.HConeComputeATimesX(g.cones[0], _p(Xs), _p(axg))
        r.L.HConeComputeATimesX(r.cones[0], _p(Xs), _p(axr))
        _close(axg, axr, 1e-11, "A X")
        _close(g.L.HConeComputeTraceCX(g.cones[0], _p(Xs)), r.L.HConeComputeTraceCX(r.cones[0], _p(Xs)), 1e-11,
               "<C, X>")
    finally:
        g.close()
        r.close()


def test_bound_and_lp_cones_match_reference(gpu_lib):
    """An SDP block with an LP cone (cone 1) and the scalar bound cone added to the KKT
    system as the reference's algorithm adds it (HKKTBuildUpExtraCone)."""
    from make_golden import lp_case
    inst, lp = lp_case("theta40+lp25")
    m, n = inst.m, inst.n
    box = np.array([-1e3, 1e3])
    blocks = [(DENSE_SDP, n, inst.Ap, inst.Ai, inst.Ax), (LP, int(lp[0]), lp[1], lp[2], lp[3]),
              (SCALAR_BOUND, 0, np.zeros(m + 2, np.int32), np.zeros(1, np.int32), box)]
    g, r = _both(blocks, m)
    try:
        y, resi, dy = probe_point(inst)
        y = np.ascontiguousarray(-np.abs(y))   # s = c - A^T y > 0 for the LP block at y <= 0
        res = {}
        for side in (g, r):
            L = side.L
            for c in side.cones:
                L.HConeSetStart(c, resi)
            flags, vals = [], []
            for c in side.cones:
                inn = C.c_int()
                assert L.HConeCheckIsInterior(c, 1.0, _p(y), C.byref(inn)) == 0
                flags.append(inn.value)
                ld = C.c_double()
                assert L.HConeGetLogBarrier(c, 0.0, None, VAR, C.byref(ld)) == 0
                st = C.c_double()
                with _quiet():
                    assert L.HConeRatioTest(c, 0.0, _p(dy), 0.5, VAR, C.byref(st)) == 0
                vals += [ld.value, st.value]
            side.init_kkt(2)
            with _quiet():
                assert L.HKKTBuildUp(side.kkt, INFEASIBLE) == 0
                assert L.HKKTBuildUpExtraCone(side.kkt, side.cones[2], INFEASIBLE) == 0
            a, ard, _, sc = side.export()
            M = np.zeros((m, m), order="F")
            if side is g:
                assert L.HKKTGetMatrix(side.kkt, _p(M)) == 0
            else:
                assert L.oracle_kkt_matrix(side.kkt, m, _p(M)) == 0
            x = np.zeros(int(lp[0]))
            L.HConeGetPrimal(side.cones[1], 0.1, _p(y), _p(np.ascontiguousarray(0.01 * dy)), _p(x), None)
            res[id(side)] = (flags, vals, a, ard, sc[3], np.tril(M), x)
        fg, vg, ag, ardg, tg, Mg, xg = res[id(g)]
        fr, vr, ar, ardr, tr, Mr, xr = res[id(r)]
        assert fg == fr
        _close(vg, vr, 1e-8, "log barriers and step bounds")
        _close(ag, ar, 1e-11, "ASinv")
        _close(ardg, ardr, 1e-11, "ASinvRdSinv")
        _close(tg, tr, 1e-11, "trace S^-1")
        _close(Mg, Mr, 1e-11, "M")
        _close(xg, xr, 1e-11, "LP x")
    finally:
        g.close()
        r.close()
