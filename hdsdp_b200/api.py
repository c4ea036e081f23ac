"""Python mirror of the reference's public C API (interface/hdsdp.h:105-116).

``Solver`` wraps one hdsdp solver object of libhdsdp_b200.so with the same
calls and argument meaning as the reference (create, init, set cone, set dual
objective, optimize, get row dual, get cone values, check solution); ``solve``
runs one ``SDPInstance`` end to end and returns the same fields as the
oracle's driver so that parity tests compare like with like.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _lib

CONETYPE_LP = 1  # HDSDP_CONETYPE_LP
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
        self._cones = {}  # cone index -> (kind, dim, user data, arrays held until optimize)

    def init(self, n_rows: int, n_cones: int = 1):
        self.m = n_rows
        return self.L.HDSDPInit(self.h, n_rows, n_cones)

    def set_cone(self, m: int, n: int, Ap, Ai, Ax):
        if len(Ap) != m + 2:
            raise ValueError("Ap must hold m + 2 column pointers (column 0 is C), got %d for m = %d" % (len(Ap), m))
        if len(Ai) < Ap[-1] or len(Ax) < Ap[-1]:
            raise ValueError("Ai / Ax shorter than Ap[m + 1]")
        Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        Ax = np.ascontiguousarray(Ax, dtype=np.float64)
        self._keep = [Ap, Ai, Ax]  # held by pointer until optimize, as in the reference
        self.n = n
        if self.L.HUserDataCreate(C.byref(self.ud)) != 0:
            raise RuntimeError("HUserDataCreate failed")
        self.L.HUserDataSetConeData(self.ud, CONETYPE_DENSE_SDP, m, n, _ip(Ap), _ip(Ai), _dp(Ax))
        return self.L.HDSDPSetCone(self.h, 0, self.ud)

    def set_lp_cone(self, m: int, n_lp: int, Ap, Ai, Ax):
        """The LP cone s = c - A^T y >= 0 as cone 1 (init with n_cones = 2): user CSC with
        m + 1 columns, column 0 the costs c, column i the coefficients of constraint i."""
        Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        Ax = np.ascontiguousarray(Ax, dtype=np.float64)
        self._keep_lp = [Ap, Ai, Ax]
        self.n_lp = n_lp
        self.ud_lp = C.c_void_p()
        if self.L.HUserDataCreate(C.byref(self.ud_lp)) != 0:
            raise RuntimeError("HUserDataCreate failed")
        self.L.HUserDataSetConeData(self.ud_lp, CONETYPE_LP, m, n_lp, _ip(Ap), _ip(Ai), _dp(Ax))
        return self.L.HDSDPSetCone(self.h, 1, self.ud_lp)

    def set_cone_at(self, i: int, kind: str, m: int, dim: int, Ap, Ai, Ax):
        """Cone ``i`` of a multi-cone problem: kind "sdp" (a block of order dim, the user CSC
        layout with packed lower-triangle rows; the library picks a dense or sparse cone)
        or "lp" (dim columns)."""
        if len(Ap) != m + 2:
            raise ValueError("Ap must hold m + 2 column pointers (column 0 is the objective)")
        arrs = [np.ascontiguousarray(Ap, dtype=np.int32), np.ascontiguousarray(Ai, dtype=np.int32),
                np.ascontiguousarray(Ax, dtype=np.float64)]
        ud = C.c_void_p()
        if self.L.HUserDataCreate(C.byref(ud)) != 0:
            raise RuntimeError("HUserDataCreate failed")
        self.L.HUserDataSetConeData(ud, CONETYPE_DENSE_SDP if kind == "sdp" else CONETYPE_LP, m, dim,
                                    _ip(arrs[0]), _ip(arrs[1]), _dp(arrs[2]))
        self._cones[i] = (kind, dim, ud, arrs)
        return self.L.HDSDPSetCone(self.h, i, ud)

    def get_cone_values_at(self, i: int):
        """(X, S) of SDP cone i (n x n), or (x, s) of LP cone i."""
        kind, dim = self._cones[i][:2]
        size = dim * dim if kind == "sdp" else dim
        P, D, aux = np.zeros(size), np.zeros(size), np.zeros(size)
        self.L.HDSDPGetConeValues(self.h, i, _dp(P), _dp(D), _dp(aux))
        if kind == "sdp":
            return P.reshape(dim, dim, order="F"), D.reshape(dim, dim, order="F")
        return P, D

    def get_lp_values(self):
        """(x, s) of the LP cone."""
        x, sl, aux = np.zeros(self.n_lp), np.zeros(self.n_lp), np.zeros(self.n_lp)
        self.L.HDSDPGetConeValues(self.h, 1, _dp(x), _dp(sl), _dp(aux))
        return x, sl

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

    def set_sparse_slack(self, mode: int):
        """Factorisation of S in the positive-definiteness checks: -1 automatic, 0 dense,
        1 sparse (minimum-degree rounds and a dense front) whenever the pattern allows."""
        self.L.HDSDPSetSparseSlack(self.h, int(mode))

    def sparse_slack_info(self) -> dict:
        o = np.zeros(8)
        self.L.HDSDPGetSparseSlackInfo(self.h, _dp(o))
        return {"cones": int(o[0]), "front": int(o[1]), "rounds": int(o[2]), "factorisations": int(o[3]),
                "eliminated": int(o[4]), "trial_factorisations": int(o[5]), "dense_after_var": int(o[6]),
                "dense_after_check": int(o[7])}

    def set_sparse_schur(self, mode: int):
        """Schur complement form when every cone is a sparse SDP cone: -1 automatic, 0 dense,
        1 block arrow (per-cone local blocks and a coupling block)."""
        self.L.HDSDPSetSparseSchur(self.h, int(mode))

    def set_schur_ldl(self, mode: int):
        """Factorisation of the dense Schur complement: 0 Cholesky (LDL^T with Bunch-Kaufman
        pivoting when the Cholesky fails even with diagonal shifts), 1 LDL^T always."""
        self.L.HDSDPSetSchurLDL(self.h, int(mode))

    def sparse_schur_info(self) -> dict:
        o = np.zeros(6)
        self.L.HDSDPGetSparseSchurInfo(self.h, _dp(o))
        return {"arrow": bool(o[0]), "coupling": int(o[1]), "cones": int(o[2]), "max_local": int(o[3]),
                "arrow_bytes": float(o[4]), "dense_bytes": float(o[5])}

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
        t = np.zeros(23)
        self.L.HDSDPGetTimers(self.h, _dp(t))
        keys = ["schur", "schur_factor", "schur_solve", "s_factor", "s_inverse", "lanczos", "assemble",
                "primal", "total", "n_schur", "n_sfactor", "n_lanczos", "n_lanczos_mv", "n_schur_solve",
                "lz_inverse", "lz_host", "lz_wait", "sch_matrix", "sch_inner", "sch_innersq", "setup",
                "ipm_device", "n_factor_reuse"]
        return dict(zip(keys, t.tolist()))

    def adjoint(self, gy=None, GX=None, want_gC=True):
        """Gradients (gb, gC, gAx) of <GX, X*> + gy^T y* after optimize() (HDSDPAdjoint)."""
        n, m = self.n, self.m
        gyv = None if gy is None else np.ascontiguousarray(gy, dtype=np.float64)
        GXf = None if GX is None else np.asfortranarray(GX, dtype=np.float64)
        gb = np.zeros(m)
        gC = np.zeros((n, n), order="F") if want_gC else None
        gAx = np.zeros(len(self._keep[2]))
        r = self.L.HDSDPAdjoint(self.h, None if gyv is None else _dp(gyv), None if GXf is None else _dp(GXf),
                                _dp(gb), None if gC is None else _dp(gC), _dp(gAx))
        if r != 0:
            raise RuntimeError("HDSDPAdjoint failed (%d)" % r)
        return gb, gC, gAx

    def close(self):
        for kind, dim, ud, arrs in self._cones.values():
            self.L.HUserDataDestroy(C.byref(ud))
        self._cones = {}
        if self.ud:
            self.L.HUserDataDestroy(C.byref(self.ud))
            if getattr(self, "ud_lp", None):
                self.L.HUserDataDestroy(C.byref(self.ud_lp))
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
          params: dict | None = None, lp=None, sparse_slack: int = -1, schur_ldl: int = 0) -> dict:
    """Solve ``inst`` on the GPU (with the LP cone ``lp`` = (n_lp, Ap, Ai, Ax) as cone 1 when
    given); returns the oracle driver's fields plus the iteration log."""
    s = Solver()
    try:
        assert s.init(inst.m, 2 if lp is not None else 1) == 0
        if s.set_cone(inst.m, inst.n, inst.Ap, inst.Ai, inst.Ax) != 0:
            raise RuntimeError("HDSDPSetCone rejected the block")
        if lp is not None and s.set_lp_cone(inst.m, int(lp[0]), lp[1], lp[2], lp[3]) != 0:
            raise RuntimeError("HDSDPSetCone rejected the LP cone")
        s.set_dual_objective(inst.b)
        s.set_primal_refinement(primal_refinement)
        s.set_precision(precision)
        s.set_sparse_slack(sparse_slack)
        s.set_schur_ldl(schur_ldl)
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
               "status": s.status(), "iters": s.iters(), "log": s.iter_log(), "timers": s.timers(),
               "sparse_slack": s.sparse_slack_info()}
        if want_x:
            X, S = s.get_cone_values()
            out["X"], out["S"] = X, S
        if lp is not None:
            out["x_lp"], out["s_lp"] = s.get_lp_values()
        out["errs"] = s.check_solution()
        out["status_after_check"] = s.status()
        return out
    finally:
        s.close()


def solve_problem(prob, primal_refinement: bool = True, precision: int = 0, params: dict | None = None,
                  sparse_slack: int = -1, sparse_schur: int = -1, schur_ldl: int = 0) -> dict:
    """Solve a multi-cone problem (instances.ConicProblem: SDP blocks and LP cones over one
    set of constraints) on the GPU; returns y, objectives, status, iterations, the iteration
    log, DIMACS errors and per cone (X, S) or (x, s)."""
    s = Solver()
    try:
        assert s.init(prob.m, len(prob.cones)) == 0
        for k, (kind, dim, Ap, Ai, Ax) in enumerate(prob.cones):
            if s.set_cone_at(k, kind, prob.m, int(dim), Ap, Ai, Ax) != 0:
                raise RuntimeError("HDSDPSetCone rejected cone %d" % k)
        s.set_dual_objective(prob.b)
        s.set_primal_refinement(primal_refinement)
        s.set_precision(precision)
        s.set_sparse_slack(sparse_slack)
        s.set_sparse_schur(sparse_schur)
        s.set_schur_ldl(schur_ldl)
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
               "status": s.status(), "iters": s.iters(), "log": s.iter_log(), "timers": s.timers(),
               "sparse_slack": s.sparse_slack_info(), "sparse_schur": s.sparse_schur_info()}
        out["values"] = [s.get_cone_values_at(k) for k in range(len(prob.cones))]
        out["errs"] = s.check_solution()
        out["status_after_check"] = s.status()
        return out
    finally:
        s.close()


# ---------------------------------------------------------------------------
# Kernel-level entry points (include/hdsdp_b200.h), host buffers in and out.

def read_sdpa_with(lib, path):
    """Call an HReadSDPA (this library's or another build of the same interface) on an SDPA
    file; returns the blocks as NumPy CSC arrays and frees the C arrays."""
    nC, nB, nCols, nLP, nE = (C.c_int() for _ in range(5))
    dims, lbeg, lidx = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    rhs, lval = C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    beg, idx = C.POINTER(C.POINTER(C.c_int))(), C.POINTER(C.POINTER(C.c_int))()
    elem = C.POINTER(C.POINTER(C.c_double))()
    outs = (nC, nB, dims, rhs, beg, idx, elem, nCols, nLP, lbeg, lidx, lval, nE)
    fn = lib.HReadSDPA
    fn.argtypes = [C.c_char_p] + [C.c_void_p] * 13
    fn.restype = C.c_int
    r = fn(str(path).encode(), *[C.addressof(x) for x in outs])
    if r != 0:
        raise RuntimeError("HReadSDPA returned %d" % r)
    free = C.CDLL(None).free
    free.argtypes = [C.c_void_p]
    m = nC.value
    blocks = []
    for k in range(nB.value):
        n = dims[k]
        Ap = np.ctypeslib.as_array(beg[k], shape=(m + 2,)).copy()
        nnz = int(Ap[-1])
        Ai = np.ctypeslib.as_array(idx[k], shape=(max(nnz, 1),))[:nnz].copy()
        Ax = np.ctypeslib.as_array(elem[k], shape=(max(nnz, 1),))[:nnz].copy()
        blocks.append((n, Ap, Ai, Ax))
        for p in (beg[k], idx[k], elem[k]):
            free(C.cast(p, C.c_void_p))
    b = np.ctypeslib.as_array(rhs, shape=(max(m, 1),))[:m].copy()
    lp = None
    if nLP.value > 0:
        Ap = np.ctypeslib.as_array(lbeg, shape=(m + 2,)).copy()
        nnz = int(Ap[-1])
        lp = (nLP.value, Ap, np.ctypeslib.as_array(lidx, shape=(max(nnz, 1),))[:nnz].copy(),
              np.ctypeslib.as_array(lval, shape=(max(nnz, 1),))[:nnz].copy())
        for p in (lbeg, lidx, lval):
            free(C.cast(p, C.c_void_p))
    for p in (dims, rhs, beg, idx, elem):
        free(C.cast(p, C.c_void_p))
    return {"m": m, "blocks": blocks, "b": b, "lp": lp, "n_cols": nCols.value, "n_elems": nE.value}


def read_sdpa(path):
    """An SDPA file through this library's HReadSDPA (include/hdsdp_file_io.h)."""
    return read_sdpa_with(_lib.load(), path)


def sdpa_cones(path):
    """An SDPA file with any number of SDP blocks and an optional LP block as a multi-cone
    problem for solve_problem(): the SDP blocks in file order, then the LP cone (the order
    the reference's own driver sets them in)."""
    from hdsdp_b200.instances import ConicProblem
    d = read_sdpa(path)
    cones = [("sdp", int(n), Ap.astype(np.int32), Ai.astype(np.int32), Ax.astype(np.float64))
             for (n, Ap, Ai, Ax) in d["blocks"]]
    if d["lp"] is not None:
        nlp, lAp, lAi, lAx = d["lp"]
        cones.append(("lp", int(nlp), lAp.astype(np.int32), lAi.astype(np.int32), lAx.astype(np.float64)))
    return ConicProblem(os.path.basename(str(path)), int(d["m"]), d["b"].astype(np.float64), cones)


def sdpa_problem(path):
    """An SDPA file with one SDP block and at most one LP block: (instance, lp) for
    solve(instance, lp=lp), lp None without an LP block."""
    from hdsdp_b200.instances import SDPInstance
    d = read_sdpa(path)
    if len(d["blocks"]) != 1:
        raise ValueError("this solver takes one SDP block (and optionally one LP block)")
    n, Ap, Ai, Ax = d["blocks"][0]
    inst = SDPInstance(os.path.basename(str(path)), n, d["m"], Ap.astype(np.int32), Ai.astype(np.int32),
                       Ax.astype(np.float64), d["b"].astype(np.float64))
    lp = None
    if d["lp"] is not None:
        nlp, lAp, lAi, lAx = d["lp"]
        lp = (nlp, lAp.astype(np.int32), lAi.astype(np.int32), lAx.astype(np.float64))
    return inst, lp


def sdpa_instance(path):
    """An SDPA file with one SDP block and no LP block as an instance for solve()."""
    from hdsdp_b200.instances import SDPInstance
    d = read_sdpa(path)
    if len(d["blocks"]) != 1 or d["lp"] is not None:
        raise ValueError("this solver takes one SDP block and no LP block")
    n, Ap, Ai, Ax = d["blocks"][0]
    return SDPInstance(os.path.basename(str(path)), n, d["m"], Ap.astype(np.int32), Ai.astype(np.int32),
                       Ax.astype(np.float64), d["b"].astype(np.float64))


def _csc(inst):
    return (np.ascontiguousarray(inst.Ap, dtype=np.int32), np.ascontiguousarray(inst.Ai, dtype=np.int32),
            np.ascontiguousarray(inst.Ax, dtype=np.float64))


def schur_probe(inst, y, resi, precision: int = 0) -> dict:
    """GPU Schur complement at S = C - A^T y - resi I (lower triangle of M, full storage)."""
    L = _lib.load()
    Ap, Ai, Ax = _csc(inst)
    y = np.ascontiguousarray(y, dtype=np.float64)
    m = inst.m
    M = np.zeros(m * m)
    asinv, asinvrd = np.zeros(m), np.zeros(m)
    tr = C.c_double()
    r = L.hdsdpb_schur_probe(m, inst.n, _ip(Ap), _ip(Ai), _dp(Ax), _dp(y), float(resi), int(precision),
                             _dp(M), _dp(asinv), _dp(asinvrd), C.byref(tr))
    if r != 0:
        raise RuntimeError("hdsdpb_schur_probe returned %d" % r)
    return {"M": np.tril(M.reshape(m, m, order="F")), "asinv": asinv, "asinvrd": asinvrd,
            "tracesinv": tr.value}


def ratio_probe(inst, y, resi, dy, ada: float):
    """GPU Lanczos step bound and log det S (first ratio test of a fresh block)."""
    L = _lib.load()
    Ap, Ai, Ax = _csc(inst)
    y = np.ascontiguousarray(y, dtype=np.float64)
    dy = np.ascontiguousarray(dy, dtype=np.float64)
    step, logdet = C.c_double(), C.c_double()
    r = L.hdsdpb_ratio_probe(inst.m, inst.n, _ip(Ap), _ip(Ai), _dp(Ax), _dp(y), float(resi), _dp(dy),
                             float(ada), C.byref(step), C.byref(logdet))
    if r != 0:
        raise RuntimeError("hdsdpb_ratio_probe returned %d" % r)
    return step.value, logdet.value


def cholesky(S):
    """(L, sum log L_ii, positive definite?) of a symmetric matrix on the GPU."""
    L = _lib.load()
    S = np.asfortranarray(S, dtype=np.float64)
    n = S.shape[0]
    out = np.zeros((n, n), order="F")
    ld = C.c_double()
    r = L.hdsdpb_cholesky(n, _dp(S), _dp(out), C.byref(ld))
    if r < 0:
        raise RuntimeError("hdsdpb_cholesky returned %d" % r)
    return out, ld.value, r == 0


def cholesky_solve(S, b):
    """x with S x = b by the Cholesky factor and blocked substitution (hdsdpb_cholesky_solve);
    None if S is not positive definite."""
    S = np.asfortranarray(S, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = S.shape[0]
    x = np.zeros(n)
    r = _lib.load().hdsdpb_cholesky_solve(n, _dp(S), _dp(b), _dp(x))
    if r < 0:
        raise RuntimeError("hdsdpb_cholesky_solve failed")
    return None if r == 1 else x


def inverse(S):
    """S^-1 of a symmetric positive definite matrix on the GPU (None if not positive definite)."""
    L = _lib.load()
    S = np.asfortranarray(S, dtype=np.float64)
    n = S.shape[0]
    out = np.zeros((n, n), order="F")
    r = L.hdsdpb_inverse(n, _dp(S), _dp(out))
    if r < 0:
        raise RuntimeError("hdsdpb_inverse returned %d" % r)
    return out if r == 0 else None


def gemm(alpha, A, B, beta=0.0, Cm=None, transA=False, transB=False):
    """alpha op(A) op(B) + beta C on the FP64 tensor-core path."""
    L = _lib.load()
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    M = A.shape[1] if transA else A.shape[0]
    K = A.shape[0] if transA else A.shape[1]
    N = B.shape[0] if transB else B.shape[1]
    Cm = np.zeros((M, N), order="F") if Cm is None else np.asfortranarray(Cm, dtype=np.float64).copy(order="F")
    r = L.hdsdpb_gemm(M, N, K, float(alpha), _dp(A), max(1, A.shape[0]), int(transA), _dp(B), max(1, B.shape[0]),
                      int(transB), float(beta), _dp(Cm), max(1, M))
    if r != 0:
        raise RuntimeError("hdsdpb_gemm returned %d" % r)
    return Cm


def split_gemm(A, B, transA=False, transB=False):
    """op(A) op(B) as BF16x3 products with FP32 accumulation on the tcgen05 tensor cores."""
    L = _lib.load()
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    M = A.shape[1] if transA else A.shape[0]
    K = A.shape[0] if transA else A.shape[1]
    N = B.shape[0] if transB else B.shape[1]
    Cm = np.zeros((M, N), order="F")
    r = L.hdsdpb_split_gemm(M, N, K, _dp(A), max(1, A.shape[0]), int(transA), _dp(B), max(1, B.shape[0]),
                            int(transB), _dp(Cm), max(1, M))
    if r != 0:
        raise RuntimeError("hdsdpb_split_gemm returned %d" % r)
    return Cm
