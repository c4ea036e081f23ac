"""Full IPM solves on the GPU against the compiled reference's results.

Parity bar: same status, iteration count within 2, objectives within 1e-6
relative, DIMACS primal/dual infeasibility within 1e-7 where the reference
reaches PRIMAL_DUAL_OPTIMAL.
"""
from __future__ import annotations

import numpy as np
import pytest

from hdsdp_b200 import api, instances
from make_golden import FULL, SMALL
from oracle import kernels_ref as K

pytestmark = pytest.mark.gpu

OPTIMAL = 3


def check_parity(r, ref, psdp=False):
    assert r["status_after_check"] == ref["status"]
    # iterations within 2 of the reference's; for long runs, of the range the reference
    # itself spans over BLAS thread counts (1 and 8 threads)
    lo, hi = ref.get("iters_range", (ref["iters"], ref["iters"]))
    assert lo - 2 <= r["iters"] <= hi + 2, (r["iters"], ref["iters"], lo, hi)
    # With primal refinement on, the dual phase stops at a 10% gap and five fixed
    # refinement steps follow. Where the reference then reaches PRIMAL_DUAL_OPTIMAL the
    # objectives meet the 1e-6 bar. Where its DIMACS check ends the run as NUMERICAL
    # (a gap of percents), the objectives keep the trajectory's floating-point drift:
    # the reference against itself with 1 and 8 BLAS threads differs by 2.7e-4 in the
    # dual objective on rank1_50_80 (tests/test_oracle_cpu.py pins that spread), so
    # those runs are held to 5e-4.
    tol = 5e-4 if (psdp and ref["status"] != OPTIMAL) else 1e-6
    assert r["dobj"] == pytest.approx(ref["dobj"], rel=tol, abs=1e-8)
    if ref["status"] == OPTIMAL:
        # a run the reference itself ends as NUMERICAL (a gap of percents) has no
        # meaningful primal objective to compare. After the five fixed refinement steps
        # the reference declares optimality at a DIMACS error up to 1e-2
        # (interface/hdsdp.c:878-895): the primal objective is then good only to the
        # run's own relative gap (err5; 1.4e-3 on theta_n300), and is held to that.
        ptol = max(tol, ref["errs"][4]) if psdp else tol
        assert r["pobj"] == pytest.approx(ref["pobj"], rel=ptol, abs=1e-8)
    if ref["status"] == OPTIMAL:
        assert r["errs"][0] <= max(1e-7, 10 * ref["errs"][0])
        assert r["errs"][1] <= 1e-7 and r["errs"][2] <= 1e-7 and r["errs"][3] <= 1e-7


@pytest.mark.parametrize("psdp", [0, 1])
@pytest.mark.parametrize("name", sorted(SMALL))
def test_small_solve_parity(gpu_lib, name, psdp, golden):
    inst = SMALL[name]()
    r = api.solve(inst, want_x=False, primal_refinement=bool(psdp))
    check_parity(r, golden["solves"]["%s/psdp%d" % (name, psdp)], psdp=bool(psdp))


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_size_parity(gpu_lib, name, golden):
    inst = FULL[name]()
    r = api.solve(inst, want_x=False, primal_refinement=False)
    check_parity(r, golden["solves"]["%s/psdp0" % name])


def test_full_size_with_primal_refinement(gpu_lib, golden):
    inst = FULL["theta_n300"]()
    r = api.solve(inst, want_x=False, primal_refinement=True)
    check_parity(r, golden["solves"]["theta_n300/psdp1"], psdp=True)


def test_known_answers(gpu_lib, golden):
    graphs = {
        "theta_C5": instances.lovasz_theta_graph(5, [(1, 0), (2, 1), (3, 2), (4, 3), (4, 0)]),
        "theta_K6": instances.lovasz_theta_graph(6, [(i, j) for i in range(6) for j in range(i)]),
        "theta_empty7": instances.lovasz_theta_graph(7, []),
    }
    for label, inst in graphs.items():
        r = api.solve(inst, want_x=False, primal_refinement=False)
        assert r["status_after_check"] == OPTIMAL, label
        assert -r["dobj"] == pytest.approx(golden["known_answers"][label]["theta"], rel=1e-7), label


def test_primal_dual_recovery(gpu_lib):
    """X and S returned by HDSDPGetConeValues satisfy the optimality conditions."""
    inst = SMALL["theta40"]()
    r = api.solve(inst, want_x=True, primal_refinement=False)
    C, A = K.dense_data(inst)
    X, S = r["X"], r["S"]
    np.testing.assert_allclose(S, K.dual_slack(C, A, r["y"]), atol=1e-9)
    e = K.dimacs(C, A, inst.b, X, S, r["y"])
    assert e[0] <= 1e-7 and e[1] <= 1e-7
    assert abs(e[2]) <= 1e-6 and abs(e[3]) <= 1e-6
    assert np.sum(C * X) == pytest.approx(r["pobj"], rel=1e-7)


@pytest.mark.slow
def test_maxcut_n8000_properties(gpu_lib):
    """MaxCut n=8000 (40000 edges): optimal with a tight duality gap, diag(X) = 1."""
    inst = instances.WORKLOADS["maxcut_n8000"]()
    r = api.solve(inst, want_x=False, primal_refinement=False)
    assert r["status_after_check"] == OPTIMAL
    assert abs(r["pobj"] - r["dobj"]) <= 1e-6 * (1 + abs(r["dobj"]))
    assert r["errs"][0] <= 1e-7
    # the SDP bound lies between half the total edge weight and the total edge weight;
    # C = -L/4 so the total weight is -2 trace(C)
    rows, vals = inst.column(0)
    i, j = K.packed_to_ij(inst.n, rows)
    total = -2.0 * np.asarray(vals)[i == j].sum()
    assert 0.5 * total <= -r["dobj"] <= total


def test_sdpa_file_solve(gpu_lib, tmp_path):
    """An instance written as an SDPA file, read back with HReadSDPA and solved, gives the
    same solve as the instance itself."""
    from test_file_io_cpu import write_sdpa
    inst = SMALL["theta40"]()
    path = tmp_path / "theta40.dat-s"
    write_sdpa(path, inst)
    via_file = api.solve(api.sdpa_instance(path), want_x=False, primal_refinement=False)
    direct = api.solve(inst, want_x=False, primal_refinement=False)
    assert via_file["status_after_check"] == direct["status_after_check"] == OPTIMAL
    assert via_file["iters"] == direct["iters"]
    assert via_file["dobj"] == pytest.approx(direct["dobj"], rel=1e-12)
    assert via_file["pobj"] == pytest.approx(direct["pobj"], rel=1e-12)


@pytest.mark.parametrize("psdp", [0, 1])
@pytest.mark.parametrize("name", ["maxcut60+lp9", "theta40+lp25", "rank1_50_80+lp31"])
def test_sdp_plus_lp_parity(gpu_lib, name, psdp, golden):
    """One SDP block with an LP cone as cone 1 (interface/hdsdp_conic_lp.c) against the
    compiled reference on the same data; with primal refinement on, the reference
    declines it for more than one cone and ends at Phase B's 10 % gap."""
    from make_golden import lp_case
    inst, lp = lp_case(name)
    r = api.solve(inst, want_x=False, primal_refinement=bool(psdp), lp=lp)
    ref = golden["lp_solves"]["%s/psdp%d" % (name, psdp)]
    check_parity(r, ref, psdp=bool(psdp))
    if ref["status"] == OPTIMAL and not psdp:
        assert r["x_lp"].min() >= -1e-7 and r["s_lp"].min() > 0.0


def test_sdpa_file_with_lp_block_solve(gpu_lib, tmp_path):
    """An SDP block plus an LP cone written as an SDPA file (diagonal LP block), read back and
    solved, matches the reference's solve of the same data."""
    from make_golden import lp_case
    from test_file_io_cpu import write_sdpa_lp
    inst, lp = lp_case("theta40+lp25")
    path = tmp_path / "theta40_lp.dat-s"
    write_sdpa_lp(path, inst, lp)
    finst, flp = api.sdpa_problem(path)
    r = api.solve(finst, want_x=False, primal_refinement=False, lp=flp)
    direct = api.solve(inst, want_x=False, primal_refinement=False, lp=lp)
    assert r["status_after_check"] == direct["status_after_check"] == OPTIMAL
    assert abs(r["iters"] - direct["iters"]) <= 2
    assert r["dobj"] == pytest.approx(direct["dobj"], rel=1e-8)


@pytest.mark.parametrize("name", sorted(instances.MULTIBLOCK_CASES))
def test_multiblock_parity(gpu_lib, name, golden, golden_arrays):
    """Several SDP blocks (dense cones, and sparse cones that build their Schur block over
    their own constraints and scatter it into M), a 1 x 1 block, and an LP cone, against
    the compiled reference on the same data (interface/hdsdp_schur.c:256-268 sums the
    cones' Schur terms in order)."""
    prob = instances.multiblock_case(name)
    r = api.solve_problem(prob)
    ref = golden["multiblock_solves"][name]
    check_parity(r, ref)
    np.testing.assert_allclose(r["y"], golden_arrays["y/" + name], rtol=1e-4, atol=1e-5)
    # each block's X is psd and the LP x nonnegative up to the DIMACS tolerance
    for (kind, _, _, _, _), (P, D) in zip(prob.cones, r["values"]):
        if kind == "sdp":
            assert np.linalg.eigvalsh(0.5 * (P + P.T)).min() > -1e-7
            assert np.linalg.eigvalsh(0.5 * (D + D.T)).min() > 0.0
        else:
            assert P.min() > -1e-7 and D.min() > 0.0


def test_multiblock_sdpa_solve(gpu_lib, tmp_path, golden):
    """A multi-block problem with an LP block written as SDPA, read back with sdpa_cones()
    and solved, matches the reference's solve of the same data."""
    from test_file_io_cpu import write_sdpa_problem
    prob = instances.multiblock_case("mb2_lp")
    path = tmp_path / "mb2_lp.dat-s"
    write_sdpa_problem(path, prob)
    r = api.solve_problem(api.sdpa_cones(path))
    check_parity(r, golden["multiblock_solves"]["mb2_lp"])

