"""Test infrastructure: counts the events of the reference's Schur-solve chain on one
workload (Jacobi-preconditioned CG, the switch to the Cholesky preconditioner, the switch to
LDL^T; linalg/hdsdp_linsolver.c:814-997, :1368-1425), from the trace of the reference built
with `make -C oracle cgtrace`.

    python oracle/cg_trace.py maxcut_n200        # a workload of hdsdp_b200.instances
    python oracle/cg_trace.py mb3                 # or a multi-block case
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from hdsdp_b200 import instances  # noqa: E402
from oracle import ref_api  # noqa: E402


def _solve(name: str) -> None:
    ref_api.LIB_PATH = os.path.join(HERE, "_ref", "libhdsdp_ref_cgtrace.so")
    if name in instances.WORKLOADS:
        r = ref_api.solve(instances.WORKLOADS[name](), want_x=False, params={4: 0}, quiet=False)
    else:
        r = ref_api.solve_problem(instances.multiblock_case(name), quiet=False)
    sys.stdout.flush()
    print("RESULT iters=%d status=%d" % (r["iters"], r["status_after_check"]), flush=True)


def main(name: str) -> dict:
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--solve", name], check=True,
                         capture_output=True, text=True).stdout
    count = lambda s: sum(1 for line in out.splitlines() if s in line)
    return {"workload": name, "jacobi_builds": count("Using Jacobi"), "cholesky_builds": count("Using Cholesky"),
            "cg_iterations": count("Conjugate iteration"), "restarts": count("restarts"),
            "switches_to_cholesky": count("switched to Cholesky"), "switches_to_ldl": count("Switch to LDL"),
            "result": [line for line in out.splitlines() if line.startswith("RESULT")][-1]}


if __name__ == "__main__":
    if sys.argv[1] == "--solve":
        _solve(sys.argv[2])
    else:
        for name in sys.argv[1:]:
            print(main(name))
