"""hdsdpb_cholesky_noalloc against the allocating entry point hdsdpb_cholesky.

The no-allocation entry point exists for callers that cannot call cudaMalloc on their
call path (their framework's allocator owns the device memory, or the allocator's
synchronisation is not acceptable there); it keeps its scratch in a static device
array. Each case is called twice in a row, because the array keeps the previous
call's contents. The file name sorts last, so in a full run it executes after every
other GPU test in the same process; it must also pass alone in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hdsdp_b200 import _lib, api

pytestmark = pytest.mark.gpu

MAX_N = 256


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.logspace(0, 3, n)) @ Q.T


def _noalloc(S):
    L = _lib.load()
    S = np.asfortranarray(S, dtype=np.float64)
    n = S.shape[0]
    out = np.zeros((n, n), order="F")
    logdiag = C.c_double()
    r = L.hdsdpb_cholesky_noalloc(n, S.ctypes.data_as(C.POINTER(C.c_double)),
                                  out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(logdiag))
    return r, out, logdiag.value


@pytest.mark.parametrize("n", [1, 37, 64, 200, MAX_N])
def test_noalloc_matches_allocating_entry(gpu_lib, n):
    S = _spd(n, n)
    Lref, ldref, pd = api.cholesky(S)
    assert pd
    Lnp = np.linalg.cholesky(S)
    for _ in range(2):
        r, L, ld = _noalloc(S)
        assert r == 0
        assert np.abs(L - Lref).max() <= 1e-12 * np.abs(Lref).max()
        assert ld == pytest.approx(ldref, rel=1e-12, abs=1e-12)
        # and against NumPy's factor directly
        assert np.abs(L - Lnp).max() <= 1e-10 * np.abs(Lnp).max()
        assert ld == pytest.approx(np.log(np.diag(Lnp)).sum(), rel=1e-10, abs=1e-10)


def test_noalloc_requests_no_buffers(gpu_lib):
    """After the first call on the device, a call makes no buffer request at all (the
    library's request counter counts its caching allocator's hits and misses alike)."""
    L = _lib.load()
    S = _spd(150, 5)
    r, _, _ = _noalloc(S)
    assert r == 0
    before = L.hdsdpb_alloc_calls()
    for _ in range(2):
        r, _, _ = _noalloc(S)
        assert r == 0
    assert L.hdsdpb_alloc_calls() == before
    # the allocating entry point does request buffers (the counter works)
    api.cholesky(S)
    assert L.hdsdpb_alloc_calls() > before


def test_noalloc_empty_matrix(gpu_lib):
    r, L, ld = _noalloc(np.zeros((0, 0)))
    assert r == 0 and ld == 0.0 and L.shape == (0, 0)


def test_noalloc_indefinite_and_size_limit(gpu_lib):
    S = _spd(50, 1)
    S[10, 10] = -1.0
    r, _, _ = _noalloc(S)
    assert r == 1
    r, _, _ = _noalloc(_spd(MAX_N + 1, 2))
    assert r == -2
    # the rejection leaves the entry point usable
    S = _spd(120, 3)
    r, L, _ = _noalloc(S)
    assert r == 0
    np.testing.assert_allclose(L @ L.T, S, rtol=0, atol=1e-10 * np.abs(S).max())
