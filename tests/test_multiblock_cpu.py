"""Multi-cone problems on the host side: the seeded generator, the cone types the library
picks for each block against the reference's HUserDataChooseCone
(interface/hdsdp_user_data.c:73-86), and the reference's own solves of the parity cases
(the golden fixtures) as a pin of the instances. No GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hdsdp_b200 import _lib, instances
from hdsdp_b200.build import build
from oracle import ref_api

OPTIMAL = 3
SPARSE_SDP, DENSE_SDP, LP = 5, 4, 1


@pytest.mark.parametrize("name", sorted(instances.MULTIBLOCK_CASES))
def test_generator(name):
    prob = instances.multiblock_case(name)
    spec = instances.MULTIBLOCK_CASES[name]
    assert prob.m == sum(spec["m_local"]) + spec["m_couple"]
    for k, (kind, n, Ap, Ai, Ax) in enumerate(prob.cones):
        assert len(Ap) == prob.m + 2
        if kind == "lp":
            assert np.all(Ax[Ap[0]:Ap[1]] > 0)  # costs c > 0: y = 0 is dual interior
            continue
        C0 = prob.sdp_block(k).dense(0)
        assert np.linalg.eigvalsh(C0).min() > 0.5  # C_k = I + small R_k
        # every coupling row touches every block
        assert np.all(np.diff(Ap)[-spec["m_couple"]:] > 0)


def _choose(L, kind, m, n, Ap, Ai, Ax):
    ud = C.c_void_p()
    assert L.HUserDataCreate(C.byref(ud)) == 0
    arrs = [np.ascontiguousarray(a) for a in (Ap, Ai, Ax)]
    L.HUserDataSetConeData(ud, DENSE_SDP if kind == "sdp" else LP, m, n,
                           arrs[0].ctypes.data_as(C.POINTER(C.c_int)), arrs[1].ctypes.data_as(C.POINTER(C.c_int)),
                           arrs[2].ctypes.data_as(C.POINTER(C.c_double)))
    t = L.HUserDataChooseCone(ud)
    L.HUserDataDestroy(C.byref(ud))
    return t


@pytest.mark.parametrize("name", sorted(instances.MULTIBLOCK_CASES))
def test_cone_choice_matches_reference(name):
    build()
    if not ref_api.available():
        pytest.skip("oracle/_ref not built")
    ours, ref = _lib.load(), ref_api.lib()
    ref.HUserDataChooseCone.argtypes = [C.c_void_p]
    prob = instances.multiblock_case(name)
    kinds = []
    for kind, n, Ap, Ai, Ax in prob.cones:
        a = _choose(ours, kind, prob.m, n, Ap, Ai, Ax)
        assert a == _choose(ref, kind, prob.m, n, Ap, Ai, Ax)
        kinds.append(a)
    if name == "mb5_sparse":
        assert kinds == [DENSE_SDP, DENSE_SDP, SPARSE_SDP, SPARSE_SDP, SPARSE_SDP]
    if name in ("mb6_sparse", "mb40_arrow"):
        assert kinds == [SPARSE_SDP] * len(prob.cones)


@pytest.mark.parametrize("name", sorted(instances.MULTIBLOCK_CASES))
def test_reference_pins(golden, name):
    """The reference solves every case to optimality with small DIMACS errors."""
    g = golden["multiblock_solves"][name]
    prob = instances.multiblock_case(name)
    assert g["m"] == prob.m and [tuple(c) for c in g["cones"]] == [(c[0], c[1]) for c in prob.cones]
    assert g["status"] == OPTIMAL
    assert max(abs(e) for e in g["errs"]) < 1e-6


def test_reference_small_case_reproduces():
    """mb5_sparse re-solved by the compiled reference gives the committed fixture."""
    if not ref_api.available():
        pytest.skip("oracle/_ref not built")
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))["multiblock_solves"]
    r = ref_api.solve_problem(instances.multiblock_case("mb5_sparse"))
    assert r["iters"] == g["mb5_sparse"]["iters"]
    assert r["dobj"] == pytest.approx(g["mb5_sparse"]["dobj"], rel=1e-12)


@pytest.mark.parametrize("m,nz", [(10, 3), (10, 4), (20, 6), (20, 7), (7, 0), (1, 1)])
def test_cone_choice_at_the_threshold(m, nz):
    """Dense when more than 0.3 m constraints have a coefficient in the block, sparse
    otherwise (interface/hdsdp_user_data.c:82-85), for the same data in both libraries."""
    build()
    if not ref_api.available():
        pytest.skip("oracle/_ref not built")
    ours, ref = _lib.load(), ref_api.lib()
    ref.HUserDataChooseCone.argtypes = [C.c_void_p]
    n = 3
    Ap = [0, 1] + [0] * m   # column 0 (C) holds one entry; then nz nonzero constraint columns
    cnt = 1
    for i in range(m):
        cnt += 1 if i < nz else 0
        Ap[i + 2] = cnt
    Ap = np.asarray(Ap, dtype=np.int32)
    Ai = np.zeros(max(cnt, 1), dtype=np.int32)
    Ax = np.ones(max(cnt, 1))
    a = _choose(ours, "sdp", m, n, Ap, Ai, Ax)
    assert a == _choose(ref, "sdp", m, n, Ap, Ai, Ax)
    assert a == (DENSE_SDP if nz > 0.3 * m else SPARSE_SDP)


def test_reference_stops_on_the_27k_row_arrow_case(golden):
    """The compiled reference's record of mb60_m27k (instances.LARGE_ARROW_CASES): it ends
    HDSDP_NUMERICAL after 26 iterations (its positive-definite sparse KKT factorisation fails
    near the optimum), with its dual objective below its primal bound."""
    g = golden["multiblock_solves"]["mb60_m27k"]
    prob = instances.multiblock_case("mb60_m27k")
    assert g["m"] == prob.m == 27100 and len(g["cones"]) == 60
    assert g["status"] == 10 and g["iters"] == 26
    assert g["dobj"] < g["pobj"]
