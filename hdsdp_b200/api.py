"""Python mirror of the reference's public C API (interface/hdsdp.h:105-116).

``Solver`` wraps one hdsdp solver object of libhdsdp_b200.so with the same
calls and argument meaning as the reference (create, init, set cone, set dual
objective, optimize, get row dual, get cone values, check solution); ``solve``
runs one ``SDPInstance`` end to end and returns the same fields as the
oracle's driver so that parity tests compare like with like.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib

CONETYPE_DENSE_SDP = 4

STATUS_NAMES = ["UNKNOWN", "DUAL_FEASIBLE", "DUAL_OPTIMAL", "PRIMAL_DUAL_OPTIMAL", "MAXITER",
                "SUSPECT_INFEAS_OR_UNBOUNDED", "INFEAS_OR_UNBOUNDED", "TIMELIMIT", "USER_INTERRUPT",
                "INTERNAL_ERROR", "NUMERICAL"]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Solver:
    """One solver object (owns a CUDA stream and its device buffers)."""

    def __init__(self):
        self.L = _lib.load()
        self.h = C.c_void_p()
        self.ud = C.c_void_p()
        if self.L.HDSDPCreate(C.byref(self.h)) != 0:
            raise RuntimeError("HDSDPCreate failed (no CUDA device?)")
        self._keep = []

    def init(self, n_rows: int, n_cones: int = 1):
        self.m = n_rows
        return self.L.HDSDPInit(self.h, n_rows, n_cones)

    def set_cone(self, m: int, n: int, Ap, Ai, Ax):
        Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        Ax = np.ascontiguousarray(Ax, dtype=np.float64)
        self._keep = [Ap, Ai, Ax]  # held by pointer until optimize, as in the reference
        self.n = n
        if self.L.HUserDataCreate(C.byref(self.ud)) != 0:
            raise RuntimeError("HUserDataCreate failed")
        self.L.HUserDataSetConeData(self.ud, CONETYPE_DENSE_SDP, m, n, _ip(Ap), _ip(Ai), _dp(Ax))
        return self.L.HDSDPSetCone(self.h, 0, self.ud)

    def set_dual_objective(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.HDSDPSetDualObjective(self.h, _dp(b))

    def set_int_param(self, k, v):
        self.L.HDSDPSetIntParam(self.h, int(k), int(v))

    def set_dbl_param(self, k, v):
        self.L.HDSDPSetDblParam(self.h, int(k), float(v))

    def set_primal_refinement(self, on: bool):
        self.L.HDSDPSetPrimalRefinement(self.h, 1 if on else 0)

    def set_precision(self, mode: int):
        self.L.HDSDPSetPrecision(self.h, int(mode))

    def optimize(self, d_only: int = 0) -> int:
        return self.L.HDSDPOptimize(self.h, int(d_only))

    def get_row_dual(self):
        y = np.zeros(self.m)
        po, do = C.c_double(), C.c_double()
        self.L.HDSDPGetRowDual(self.h, C.byref(po), C.byref(do), _dp(y))
        return po.value, do.value, y

    def get_cone_values(self):
        n = self.n
        X = np.zeros(n * n)
        S = np.zeros(n * n)
        aux = np.zeros(n * n)
        self.L.HDSDPGetConeValues(self.h, 0, _dp(X), _dp(S), _dp(aux))
        return X.reshape(n, n, order="F"), S.reshape(n, n, order="F")

    def check_solution(self):
        e = np.zeros(6)
        self.L.HDSDPCheckSolution(self.h, _dp(e))
        return e

    def status(self) -> int:
        return self.L.HDSDPGetStatus(self.h)

    def iters(self) -> int:
        return self.L.HDSDPGetIterCount(self.h)

    def iter_log(self):
        k = self.L.HDSDPGetIterLog(self.h, 0, None, None, None, None, None, None)
        arr = {key: np.zeros(k) for key in ("t", "pobj", "dobj", "mu", "gap")}
        ph = np.zeros(k, dtype=np.int32)
        self.L.HDSDPGetIterLog(self.h, k, _dp(arr["t"]), _dp(arr["pobj"]), _dp(arr["dobj"]),
                               _dp(arr["mu"]), _dp(arr["gap"]), _ip(ph))
        arr["phase"] = ph
        return arr

    def timers(self):
        t = np.zeros(20)
        self.L.HDSDPGetTimers(self.h, _dp(t))
        keys = ["schur", "schur_factor", "schur_solve", "s_factor", "s_inverse", "lanczos", "assemble",
                "primal", "total", "n_schur", "n_sfactor", "n_lanczos", "n_lanczos_mv", "n_schur_solve",
                "lz_inverse", "lz_host", "lz_wait", "sch_matrix", "sch_inner", "sch_innersq"]
        return dict(zip(keys, t.tolist()))

    def close(self):
        if self.ud:
            self.L.HUserDataDestroy(C.byref(self.ud))
            self.ud = C.c_void_p()
        if self.h:
            self.L.HDSDPDestroy(C.byref(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve(inst, want_x: bool = True, primal_refinement: bool = True, precision: int = 0,
          params: dict | None = None) -> dict:
    """Solve ``inst`` on the GPU; returns the oracle driver's fields plus the iteration log."""
    s = Solver()
    try:
        assert s.init(inst.m, 1) == 0
        if s.set_cone(inst.m, inst.n, inst.Ap, inst.Ai, inst.Ax) != 0:
            raise RuntimeError("HDSDPSetCone rejected the block")
        s.set_dual_objective(inst.b)
        s.set_primal_refinement(primal_refinement)
        s.set_precision(precision)
        for k, v in (params or {}).items():
            if isinstance(v, int):
                s.set_int_param(k, v)
            else:
                s.set_dbl_param(k, v)
        t0 = time.perf_counter()
        ret = s.optimize(0)
        t1 = time.perf_counter()
        po, do, y = s.get_row_dual()
        out = {"retcode": int(ret), "time": t1 - t0, "y": y, "pobj": po, "dobj": do,
               "status": s.status(), "iters": s.iters(), "log": s.iter_log(), "timers": s.timers()}
        if want_x:
            X, S = s.get_cone_values()
            out["X"], out["S"] = X, S
        out["errs"] = s.check_solution()
        out["status_after_check"] = s.status()
        return out
    finally:
        s.close()
