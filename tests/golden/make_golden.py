"""Generate the golden fixtures of tests/ by running the compiled reference.

    make -C oracle && python tests/golden/make_golden.py [--full]
    python tests/golden/make_golden.py --add GROUP [GROUP ...]

--add runs only the named groups (EXTRA below) and merges their results into
the existing fixtures: "maxcut_theta" (MaxCut n=8000 and the theta layer n=200,
primal refinement off; a few minutes), "stock" (the sparse-dual instances on
the reference build with its own dual-storage rule), "hsd" (instances that end
in the homogeneous self-dual embedding), "dense" (general dense coefficients),
"multiblock" (multi-cone cases missing from the fixtures), "large" (the 60-cone
m = 27,100 block-arrow case; about half an hour on 8 cores, most of it the reference's
dense stand-in for its sparse KKT factorisation).

Writes tests/golden/golden.json (solver results and probe outputs) and
tests/golden/golden_arrays.npz (Schur matrices, dual vectors). The inputs are
the seeded instances of hdsdp_b200/instances.py, so the same arrays are
regenerated bit-for-bit wherever the tests run. --full also solves the
full-size Lovasz-theta (n=300) and rank-one (n=1000, m=2000) workloads
(about two minutes of CPU time with the reference).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hdsdp_b200 import instances  # noqa: E402
from oracle import ref_api  # noqa: E402

# Small cases that the parity tests solve on every run.
SMALL = {
    "maxcut60": lambda: instances.maxcut(60, 0.1, seed=11),
    "maxcut200": lambda: instances.maxcut(200, 0.05, seed=1),
    "theta40": lambda: instances.lovasz_theta(40, 0.2, seed=3),
    "rank1_50_80": lambda: instances.rank_one(50, 80, 0.2, seed=4),
    "theta_adj40": lambda: instances.theta_adjoint(40, 0.2, 0.3, seed=2),
}
# The small SDP blocks with an LP cone as cone 1 (instances.lp_block).
LP_CASES = {
    "maxcut60+lp9": ("maxcut60", 9, 2, 11),
    "theta40+lp25": ("theta40", 25, 2, 12),
    "rank1_50_80+lp31": ("rank1_50_80", 31, 3, 13),
}


def lp_case(name):
    base, nlp, per, seed = LP_CASES[name]
    inst = SMALL[base]()
    return inst, instances.lp_block(inst.m, nlp, per, seed=seed)


FULL = {
    "theta_n300": lambda: instances.WORKLOADS["theta_n300"](),
    "rank1_n1000_m2000": lambda: instances.WORKLOADS["rank1_n1000_m2000"](),
}


# Groups generated on demand (--add) and merged into the fixtures.
MAXCUT_THETA = {
    "maxcut_n8000": lambda: instances.WORKLOADS["maxcut_n8000"](),
    "theta_adjoint_n200": lambda: instances.WORKLOADS["theta_adjoint_n200"](),
}
STOCK = {
    "maxcut60": SMALL["maxcut60"],
    "maxcut200": SMALL["maxcut200"],
    "theta_adj40": SMALL["theta_adj40"],
    "theta_adjoint_n200": MAXCUT_THETA["theta_adjoint_n200"],
    "maxcut_n8000": MAXCUT_THETA["maxcut_n8000"],
}
HSD = {
    "dinf8": lambda: instances.dual_infeasible(8, seed=1),
    "dinf30": lambda: instances.dual_infeasible(30, seed=2),
}
# primal refinement on is not generated: the reference's PSDP asserts on dense
# coefficients (linalg/hdsdp_sdpdata.c:1963)
DENSE = {
    "dense40": lambda: instances.dense_coeff(40, 20, seed=22),
    "dense80": lambda: instances.dense_coeff(80, 40, seed=21),
}


def _solve_record(inst, r):
    return {"n": inst.n, "m": inst.m, "retcode": r["retcode"], "iters": r["iters"],
            "status": r["status_after_check"], "status_before_check": r["status"], "pobj": r["pobj"],
            "dobj": r["dobj"], "errs": [float(e) for e in r["errs"]], "time_s": r["time"]}


def add_groups(groups):
    """Run the named groups and merge their results into the committed fixtures."""
    gpath, apath = os.path.join(HERE, "golden.json"), os.path.join(HERE, "golden_arrays.npz")
    out = json.load(open(gpath))
    arrays = dict(np.load(apath))
    for g in groups:
        if g == "maxcut_theta":
            for name, make in MAXCUT_THETA.items():
                inst = make()
                r = ref_api.solve(inst, want_x=False, params={4: 0})
                key = "%s/psdp0" % name
                out["solves"][key] = _solve_record(inst, r)
                arrays["y/" + key] = r["y"]
                print(key, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], r["time"], flush=True)
        elif g == "stock":
            out.setdefault("solves_stock", {})
            for name, make in STOCK.items():
                inst = make()
                r = ref_api.solve(inst, want_x=False, params={4: 0}, variant="stock")
                key = "%s/psdp0" % name
                out["solves_stock"][key] = _solve_record(inst, r)
                arrays["y_stock/" + key] = r["y"]
                print("stock", key, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], r["time"], flush=True)
        elif g == "hsd":
            out.setdefault("hsd_solves", {})
            for name, make in HSD.items():
                inst = make()
                for psdp in (0, 1):
                    r = ref_api.solve(inst, want_x=False, params={4: psdp})
                    key = "%s/psdp%d" % (name, psdp)
                    out["hsd_solves"][key] = _solve_record(inst, r)
                    print("hsd", key, r["iters"], r["status"], r["status_after_check"], r["pobj"], r["dobj"], flush=True)
        elif g == "multiblock":
            # multi-cone cases not yet in the fixtures
            for name in instances.MULTIBLOCK_CASES:
                rec = out.get("multiblock_solves", {}).get(name)
                if rec is not None:
                    if instances.multiblock_case(name).m >= 4096 and "iters_range" not in rec:
                        # long runs: the reference's own iteration count depends on its BLAS
                        # thread count (fixed when OpenBLAS loads); record the count of a
                        # one-thread run in a child process beside the default
                        import subprocess
                        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
                        it1 = int(subprocess.run([sys.executable, os.path.abspath(__file__), "--iters", name],
                                                 env=env, check=True, capture_output=True,
                                                 text=True).stdout.strip().splitlines()[-1])
                        rec["iters_range"] = [min(rec["iters"], it1), max(rec["iters"], it1)]
                        print("multiblock", name, "one thread:", it1, flush=True)
                    continue
                prob = instances.multiblock_case(name)
                r = ref_api.solve_problem(prob)
                out["multiblock_solves"][name] = {
                    "m": prob.m, "cones": [[c[0], int(c[1])] for c in prob.cones], "retcode": r["retcode"],
                    "iters": r["iters"], "status": r["status_after_check"], "pobj": r["pobj"], "dobj": r["dobj"],
                    "errs": [float(e) for e in r["errs"]],
                }
                arrays["y/" + name] = r["y"]
                print("multiblock", name, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], flush=True)
        elif g == "large":
            # the large block-arrow case that the reference can still solve here (its sparse KKT
            # through the dense stand-in: a 5.9 GB M and a dense factorisation per iteration)
            out.setdefault("multiblock_solves", {})
            for name in ("mb60_m27k",):
                if name in out["multiblock_solves"]:
                    continue
                prob = instances.multiblock_case(name)
                r = ref_api.solve_problem(prob)
                out["multiblock_solves"][name] = {
                    "m": prob.m, "cones": [[c[0], int(c[1])] for c in prob.cones], "retcode": r["retcode"],
                    "iters": r["iters"], "status": r["status_after_check"], "pobj": r["pobj"], "dobj": r["dobj"],
                    "errs": [float(e) for e in r["errs"]],
                }
                arrays["y/" + name] = r["y"]
                print("large", name, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], flush=True)
        elif g == "dense":
            out.setdefault("dense_solves", {})
            for name, make in DENSE.items():
                inst = make()
                r = ref_api.solve(inst, want_x=False, params={4: 0})
                key = "%s/psdp0" % name
                out["dense_solves"][key] = _solve_record(inst, r)
                arrays["y/" + key] = r["y"]
                print("dense", key, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], flush=True)
                y, resi, dy = probe_point(inst)
                sp = ref_api.schur_probe(inst, y, resi)
                step, logdet = ref_api.ratio_probe(inst, y, resi, dy, 0.5)
                out["probes"][name] = {"resi": resi, "tracesinv": sp["tracesinv"], "step": step, "logdet": logdet}
                arrays["M/" + name] = np.tril(sp["M"])
                arrays["asinv/" + name] = sp["asinv"]
                arrays["asinvrd/" + name] = sp["asinvrd"]
        else:
            raise SystemExit("unknown group %s" % g)
        json.dump(out, open(gpath, "w"), indent=1, sort_keys=True)
        np.savez_compressed(apath, **arrays)


def probe_point(inst, seed=0):
    rng = np.random.default_rng(seed)
    y = -np.abs(rng.standard_normal(inst.m)) * 0.1
    resi = -(inst.n + 10.0)
    dy = rng.standard_normal(inst.m)
    return y, resi, dy


def main(full: bool):
    out = {"solves": {}, "probes": {}}
    arrays = {}
    cases = dict(SMALL)
    if full:
        cases.update(FULL)
    for name, make in cases.items():
        inst = make()
        for psdp in (0, 1):
            r = ref_api.solve(inst, want_x=False, params={4: psdp})
            key = "%s/psdp%d" % (name, psdp)
            out["solves"][key] = {
                "n": inst.n, "m": inst.m, "retcode": r["retcode"], "iters": r["iters"],
                "status": r["status_after_check"], "pobj": r["pobj"], "dobj": r["dobj"],
                "errs": [float(e) for e in r["errs"]], "time_s": r["time"],
            }
            arrays["y/" + key] = r["y"]
            print(key, out["solves"][key]["iters"], out["solves"][key]["status"], r["pobj"], r["dobj"], flush=True)
        if name in SMALL:
            y, resi, dy = probe_point(inst)
            sp = ref_api.schur_probe(inst, y, resi)
            step, logdet = ref_api.ratio_probe(inst, y, resi, dy, 0.5)
            out["probes"][name] = {"resi": resi, "tracesinv": sp["tracesinv"], "step": step, "logdet": logdet}
            arrays["M/" + name] = np.tril(sp["M"])
            arrays["asinv/" + name] = sp["asinv"]
            arrays["asinvrd/" + name] = sp["asinvrd"]
    # SDP block + LP cone
    out["lp_solves"] = {}
    for name in LP_CASES:
        inst, lp = lp_case(name)
        for psdp in (0, 1):
            r = ref_api.solve(inst, want_x=False, params={4: psdp}, lp=lp)
            key = "%s/psdp%d" % (name, psdp)
            out["lp_solves"][key] = {
                "n": inst.n, "m": inst.m, "n_lp": int(lp[0]), "retcode": r["retcode"], "iters": r["iters"],
                "status": r["status_after_check"], "pobj": r["pobj"], "dobj": r["dobj"],
                "errs": [float(e) for e in r["errs"]],
            }
            arrays["y/" + key] = r["y"]
            arrays["x_lp/" + key] = r["x_lp"]
            print(key, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], flush=True)
    # several cones: SDP blocks (dense and sparse cones, a 1 x 1 block) and an LP cone
    out["multiblock_solves"] = {}
    for name in instances.MULTIBLOCK_CASES:
        prob = instances.multiblock_case(name)
        r = ref_api.solve_problem(prob)
        out["multiblock_solves"][name] = {
            "m": prob.m, "cones": [[c[0], int(c[1])] for c in prob.cones], "retcode": r["retcode"],
            "iters": r["iters"], "status": r["status_after_check"], "pobj": r["pobj"], "dobj": r["dobj"],
            "errs": [float(e) for e in r["errs"]],
        }
        arrays["y/" + name] = r["y"]
        print(name, r["iters"], r["status_after_check"], r["pobj"], r["dobj"], flush=True)
    # known answers of the Lovasz theta number, solved by the reference
    ka = {}
    for label, inst, value in [
        ("theta_C5", instances.lovasz_theta_graph(5, [(1, 0), (2, 1), (3, 2), (4, 3), (4, 0)]), np.sqrt(5.0)),
        ("theta_K6", instances.lovasz_theta_graph(6, [(i, j) for i in range(6) for j in range(i)]), 1.0),
        ("theta_empty7", instances.lovasz_theta_graph(7, []), 7.0),
    ]:
        r = ref_api.solve(inst, want_x=False, params={4: 0})
        ka[label] = {"theta": value, "ref_dobj": r["dobj"], "ref_status": r["status_after_check"]}
        print(label, value, r["dobj"], flush=True)
    out["known_answers"] = ka
    if not full:
        old = os.path.join(HERE, "golden.json")
        if os.path.exists(old):
            prev = json.load(open(old))
            for k, v in prev.get("solves", {}).items():
                if k.split("/")[0] in FULL:
                    out["solves"][k] = v
            prevarr = np.load(os.path.join(HERE, "golden_arrays.npz"))
            for k in prevarr.files:
                if k.split("/")[1] in FULL:
                    arrays[k] = prevarr[k]
    json.dump(out, open(os.path.join(HERE, "golden.json"), "w"), indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "golden_arrays.npz"), **arrays)


if __name__ == "__main__":
    if "--iters" in sys.argv:
        # iteration count of the reference's solve of one multi-block case (last line)
        r = ref_api.solve_problem(instances.multiblock_case(sys.argv[sys.argv.index("--iters") + 1]))
        print(r["iters"])
    elif "--add" in sys.argv:
        add_groups(sys.argv[sys.argv.index("--add") + 1:])
    else:
        main("--full" in sys.argv)
