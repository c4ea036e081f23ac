"""Build libhdsdp_b200.so in-tree with nvcc for sm_100a.

    python -m hdsdp_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libhdsdp_b200.so")
SOURCES = ["la.cu", "chol.cu", "sdp.cu", "split.cu", "cone.cu", "solver.cu", "ext.cu", "adjoint.cu", "noalloc.cu", "lp.cu", "conic.cu", "sparse_chol.cu", "arrow.cu", "ldl.cu", "file_io.cpp"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "-shared", "-cudart", "static", "-diag-suppress", "550",
              "-lgomp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def build(force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".cpp"))]
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in deps):
            return OUT
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", OUT] + srcs
    subprocess.run(cmd, check=True, cwd=CSRC)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
