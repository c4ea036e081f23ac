"""The C-ABI library without a GPU: it builds, loads, exports every declared
entry point, and refuses to run on the CPU."""
from __future__ import annotations

import ast
import glob
import os
import re

import pytest

from hdsdp_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"extern\s+[\w\s\*]+?\b(\w+)\s*\(", src):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.load()


def test_headers_match_binding_list():
    assert declared_functions() == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing


def test_no_cpu_path(lib):
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert lib.HDSDPCreate(C.byref(h)) != 0
    assert not h.value


def test_user_data_host_logic(lib):
    """HUserData* is host-only bookkeeping (interface/hdsdp_user_data.c)."""
    import ctypes as C
    import numpy as np
    ud = C.c_void_p()
    assert lib.HUserDataCreate(C.byref(ud)) == 0
    Ap = np.array([0, 1, 2], dtype=np.int32)
    Ai = np.array([0, 2], dtype=np.int32)
    Ax = np.array([1.0, 1.0])
    lib.HUserDataSetConeData(ud, 4, 1, 2, Ap.ctypes.data_as(C.POINTER(C.c_int)),
                             Ai.ctypes.data_as(C.POINTER(C.c_int)), Ax.ctypes.data_as(C.POINTER(C.c_double)))
    assert lib.HUserDataChooseCone(ud) == 4  # HDSDP_CONETYPE_DENSE_SDP
    lib.HUserDataDestroy(C.byref(ud))
    assert not ud.value


def test_product_never_imports_the_oracle():
    for path in glob.glob(os.path.join(ROOT, "hdsdp_b200", "*.py")):
        tree = ast.parse(open(path).read())
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                mods = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                mods = [node.module or ""]
            else:
                continue
            assert not any(m.split(".")[0] == "oracle" for m in mods), path
