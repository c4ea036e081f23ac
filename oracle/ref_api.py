"""ctypes driver for the reference HDSDP solver built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY. Imported by tests/ (parity checks, golden vectors)
and by bench.py's reference / CPU-baseline arm; never by the product package.

It feeds an ``SDPInstance`` through the reference's public C API
(interface/hdsdp.h:105-116, interface/hdsdp_user_data.h:18-23) exactly as a C
caller would, and reads status / iteration count through oracle/ref_probe.c.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libhdsdp_ref.so")
# The same sources built with the reference's own dual-storage rule (sparse CSC below 25 %
# fill, interface/hdsdp_conic_sdp.c:33-35, :94); usable with primal refinement off only.
LIB_PATH_STOCK = os.path.join(HERE, "_ref", "libhdsdp_ref_stock.so")

CONETYPE_LP = 1  # HDSDP_CONETYPE_LP
CONETYPE_DENSE_SDP = 4  # interface/def_hdsdp_conic.h:22-32

_libs = {}


def _path(variant: str) -> str:
    return {"dense": LIB_PATH, "stock": LIB_PATH_STOCK}[variant]


def available(variant: str = "dense") -> bool:
    return os.path.exists(_path(variant))


def lib(variant: str = "dense"):
    if variant not in _libs:
        if not available(variant):
            raise RuntimeError("reference oracle not built: run `make -C oracle` where the reference tree exists")
        L = C.CDLL(_path(variant))
        vp = C.c_void_p
        L.HDSDPCreate.argtypes = [C.POINTER(vp)]
        L.HDSDPInit.argtypes = [vp, C.c_int, C.c_int]
        L.HDSDPSetCone.argtypes = [vp, C.c_int, vp]
        L.HDSDPSetDualObjective.argtypes = [vp, C.POINTER(C.c_double)]
        L.HDSDPOptimize.argtypes = [vp, C.c_int]
        L.HDSDPSetIntParam.argtypes = [vp, C.c_int, C.c_int]
        L.HDSDPSetDblParam.argtypes = [vp, C.c_int, C.c_double]
        L.HDSDPGetRowDual.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.HDSDPGetConeValues.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.HDSDPCheckSolution.argtypes = [vp, C.POINTER(C.c_double)]
        L.HDSDPDestroy.argtypes = [C.POINTER(vp)]
        L.HUserDataCreate.argtypes = [C.POINTER(vp)]
        L.HUserDataSetConeData.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.HUserDataDestroy.argtypes = [C.POINTER(vp)]
        L.oracle_status.argtypes = [vp]
        L.oracle_iters.argtypes = [vp]
        L.oracle_perturb.argtypes = [vp]
        L.oracle_perturb.restype = C.c_double
        L.oracle_mu.argtypes = [vp]
        L.oracle_mu.restype = C.c_double
        L.oracle_int_param.argtypes = [vp, C.c_int]
        L.oracle_dbl_param.argtypes = [vp, C.c_int]
        L.oracle_set_int_param.argtypes = [vp, C.c_int, C.c_int]
        L.oracle_dbl_param.restype = C.c_double
        L.oracle_schur_probe.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                         C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
        L.oracle_ratio_probe.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                         C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
        _libs[variant] = L
    return _libs[variant]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def set_threads(n: int):
    """Thread count of the BLAS under the reference (MKL stand-in)."""
    try:
        L = C.CDLL(LIB_PATH)
        L.MKL_Set_Num_Threads(int(n))
    except OSError:
        pass


def solve(inst, want_x: bool = True, params: dict | None = None, quiet: bool = True, lp=None,
          variant: str = "dense") -> dict:
    """Run HDSDPOptimize on ``inst`` (plus the LP cone ``lp`` = (n_lp, Ap, Ai, Ax) as cone 1,
    as the reference's own driver adds it); return y, objectives, status, X, S, errors, time.
    ``variant`` "stock" runs the build with the reference's own dual-storage rule."""
    L = lib(variant)
    Ap = np.ascontiguousarray(inst.Ap, dtype=np.int32)
    Ai = np.ascontiguousarray(inst.Ai, dtype=np.int32)
    Ax = np.ascontiguousarray(inst.Ax, dtype=np.float64)
    b = np.ascontiguousarray(inst.b, dtype=np.float64)
    h = C.c_void_p()
    ud = C.c_void_p()
    assert L.HDSDPCreate(C.byref(h)) == 0
    assert L.HUserDataCreate(C.byref(ud)) == 0
    L.HUserDataSetConeData(ud, CONETYPE_DENSE_SDP, inst.m, inst.n, _ip(Ap), _ip(Ai), _dp(Ax))
    ulp = C.c_void_p()
    keep = []
    assert L.HDSDPInit(h, inst.m, 2 if lp is not None else 1) == 0
    assert L.HDSDPSetCone(h, 0, ud) == 0
    if lp is not None:
        nlp, lAp, lAi, lAx = lp
        keep = [np.ascontiguousarray(lAp, dtype=np.int32), np.ascontiguousarray(lAi, dtype=np.int32),
                np.ascontiguousarray(lAx, dtype=np.float64)]
        assert L.HUserDataCreate(C.byref(ulp)) == 0
        L.HUserDataSetConeData(ulp, CONETYPE_LP, inst.m, int(nlp), _ip(keep[0]), _ip(keep[1]), _dp(keep[2]))
        assert L.HDSDPSetCone(h, 1, ulp) == 0
    L.HDSDPSetDualObjective(h, _dp(b))
    for k, v in (params or {}).items():
        if isinstance(v, int):
            if k >= 3:
                L.oracle_set_int_param(h, k, v)
            else:
                L.HDSDPSetIntParam(h, k, v)
        else:
            L.HDSDPSetDblParam(h, k, float(v))
    saved = None
    if quiet:
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)
    try:
        t0 = time.perf_counter()
        ret = L.HDSDPOptimize(h, 0)
        t1 = time.perf_counter()
        y = np.zeros(inst.m)
        po, do = C.c_double(), C.c_double()
        L.HDSDPGetRowDual(h, C.byref(po), C.byref(do), _dp(y))
        out = {"retcode": int(ret), "time": t1 - t0, "y": y, "pobj": po.value, "dobj": do.value,
               "status": int(L.oracle_status(h)), "iters": int(L.oracle_iters(h)),
               "perturb": float(L.oracle_perturb(h))}
        if want_x:
            n = inst.n
            X = np.zeros(n * n)
            S = np.zeros(n * n)
            aux = np.zeros(n * n)
            L.HDSDPGetConeValues(h, 0, _dp(X), _dp(S), _dp(aux))
            out["X"] = X.reshape(n, n, order="F")
            out["S"] = S.reshape(n, n, order="F")
        errs = np.zeros(6)
        L.HDSDPCheckSolution(h, _dp(errs))
        out["errs"] = errs
        out["status_after_check"] = int(L.oracle_status(h))
        if lp is not None:
            xl, sl = np.zeros(int(lp[0])), np.zeros(int(lp[0]))
            L.HDSDPGetConeValues(h, 1, _dp(xl), _dp(sl), _dp(np.zeros(int(lp[0]))))
            out["x_lp"], out["s_lp"] = xl, sl
            L.HUserDataDestroy(C.byref(ulp))
        L.HUserDataDestroy(C.byref(ud))
        L.HDSDPDestroy(C.byref(h))  # prints its closing line
    finally:
        if quiet:
            import sys
            sys.stdout.flush()
            C.CDLL(None).fflush(None)  # C stdio buffers of the reference's log
            os.dup2(saved, 1)
            os.close(saved)
    return out


def solve_problem(prob, params: dict | None = None, quiet: bool = True) -> dict:
    """Run HDSDPOptimize on a multi-cone ``prob`` (instances.ConicProblem): every cone set in
    its order through HDSDPSetCone (SDP blocks as dense SDP user data, the reference choosing
    dense or sparse cones itself; LP cones as LP). Returns y, objectives, status, iterations,
    DIMACS errors and per cone (X, S) or (x, s)."""
    L = lib()
    h = C.c_void_p()
    assert L.HDSDPCreate(C.byref(h)) == 0
    assert L.HDSDPInit(h, prob.m, len(prob.cones)) == 0
    keep, uds = [], []
    for k, (kind, dim, Ap, Ai, Ax) in enumerate(prob.cones):
        arrs = [np.ascontiguousarray(Ap, dtype=np.int32), np.ascontiguousarray(Ai, dtype=np.int32),
                np.ascontiguousarray(Ax, dtype=np.float64)]
        keep.append(arrs)
        ud = C.c_void_p()
        assert L.HUserDataCreate(C.byref(ud)) == 0
        L.HUserDataSetConeData(ud, CONETYPE_DENSE_SDP if kind == "sdp" else CONETYPE_LP, prob.m, int(dim),
                               _ip(arrs[0]), _ip(arrs[1]), _dp(arrs[2]))
        uds.append(ud)
        assert L.HDSDPSetCone(h, k, ud) == 0
    b = np.ascontiguousarray(prob.b, dtype=np.float64)
    L.HDSDPSetDualObjective(h, _dp(b))
    for k, v in (params or {}).items():
        if isinstance(v, int):
            if k >= 3:
                L.oracle_set_int_param(h, k, v)
            else:
                L.HDSDPSetIntParam(h, k, v)
        else:
            L.HDSDPSetDblParam(h, k, float(v))
    saved = None
    if quiet:
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)
    try:
        t0 = time.perf_counter()
        ret = L.HDSDPOptimize(h, 0)
        t1 = time.perf_counter()
        y = np.zeros(prob.m)
        po, do = C.c_double(), C.c_double()
        L.HDSDPGetRowDual(h, C.byref(po), C.byref(do), _dp(y))
        out = {"retcode": int(ret), "time": t1 - t0, "y": y, "pobj": po.value, "dobj": do.value,
               "status": int(L.oracle_status(h)), "iters": int(L.oracle_iters(h))}
        values = []
        for k, (kind, dim, _, _, _) in enumerate(prob.cones):
            size = dim * dim if kind == "sdp" else dim
            P, D, aux = np.zeros(size), np.zeros(size), np.zeros(size)
            L.HDSDPGetConeValues(h, k, _dp(P), _dp(D), _dp(aux))
            if kind == "sdp":
                P, D = P.reshape(dim, dim, order="F"), D.reshape(dim, dim, order="F")
            values.append((P, D))
        out["values"] = values
        errs = np.zeros(6)
        L.HDSDPCheckSolution(h, _dp(errs))
        out["errs"] = errs
        out["status_after_check"] = int(L.oracle_status(h))
        for ud in uds:
            L.HUserDataDestroy(C.byref(ud))
        L.HDSDPDestroy(C.byref(h))
    finally:
        if quiet:
            import sys
            sys.stdout.flush()
            C.CDLL(None).fflush(None)
            os.dup2(saved, 1)
            os.close(saved)
    return out


def schur_probe(inst, y, resi, type_kkt: int = 0):
    """Reference Schur complement at (y, resi): returns dict(M lower, asinv, asinvrd, ...)."""
    L = lib()
    m, n = inst.m, inst.n
    Ap = np.ascontiguousarray(inst.Ap, dtype=np.int32)
    Ai = np.ascontiguousarray(inst.Ai, dtype=np.int32)
    Ax = np.ascontiguousarray(inst.Ax, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    M = np.zeros(m * m)
    asinv = np.zeros(m)
    asinvrd = np.zeros(m)
    asinvcs = np.zeros(m)
    scal = np.zeros(4)
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    os.close(devnull)
    try:
        r = L.oracle_schur_probe(m, n, _ip(Ap), _ip(Ai), _dp(Ax), _dp(y), float(resi), int(type_kkt),
                                 _dp(M), _dp(asinv), _dp(asinvrd), _dp(asinvcs), _dp(scal))
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
    if r != 0:
        raise RuntimeError("schur probe failed (%d)" % r)
    return {"M": M.reshape(m, m, order="F"), "asinv": asinv, "asinvrd": asinvrd,
            "asinvcs": asinvcs, "csinv": scal[0], "csinvcsinv": scal[1], "csinvrd": scal[2],
            "tracesinv": scal[3]}


def ratio_probe(inst, y, resi, dy, ada):
    """Reference Lanczos step bound for S(y) + alpha dS(dy) (first call of a fresh cone)."""
    L = lib()
    Ap = np.ascontiguousarray(inst.Ap, dtype=np.int32)
    Ai = np.ascontiguousarray(inst.Ai, dtype=np.int32)
    Ax = np.ascontiguousarray(inst.Ax, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    dy = np.ascontiguousarray(dy, dtype=np.float64)
    step = C.c_double()
    logdet = C.c_double()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    os.close(devnull)
    try:
        r = L.oracle_ratio_probe(inst.m, inst.n, _ip(Ap), _ip(Ai), _dp(Ax), _dp(y), float(resi),
                                 _dp(dy), float(ada), C.byref(step), C.byref(logdet))
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
    if r != 0:
        raise RuntimeError("ratio probe failed (%d)" % r)
    return step.value, logdet.value
