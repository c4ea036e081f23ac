"""The FP64 adjoint restatement against central finite differences of the
compiled reference solver (CPU only).

The loss is L = <G, X*> + h^T y* with G symmetric Gaussian and h Gaussian;
the data directions are random perturbations of C's stored values and of b.
The reference solves to a relative gap of about 1e-9, so with a step of 1e-5
the finite differences carry an error of a few 1e-3 relative.
"""
from __future__ import annotations

import copy

import numpy as np
import pytest

from hdsdp_b200 import instances
from oracle import adjoint_ref, ref_api

pytestmark = pytest.mark.skipif(not ref_api.available(), reason="oracle/_ref not built (make -C oracle)")


def _solve(inst, Ax, b):
    I = copy.copy(inst)
    I.Ax, I.b = Ax, b
    return ref_api.solve(I, want_x=True, params={4: 0})


@pytest.mark.parametrize("make", [lambda: instances.maxcut(30, 0.3, seed=3),
                                  lambda: instances.rank_one(20, 30, 0.3, seed=6)])
def test_adjoint_matches_finite_differences(make):
    inst = make()
    r0 = _solve(inst, inst.Ax.copy(), inst.b.copy())
    assert r0["status_after_check"] == 3
    rng = np.random.default_rng(1)
    n, m = inst.n, inst.m
    G = rng.standard_normal((n, n))
    G = G + G.T
    h = rng.standard_normal(m)
    gb, gC, gAx = adjoint_ref.vjp(inst, r0["y"], r0["X"], h, G)

    def loss(r):
        return float(np.sum(G * r["X"]) + h @ r["y"])

    eps = 1e-5
    for _ in range(3):
        dAx = np.zeros(inst.Ax.size)
        dAx[:inst.Ap[1]] = rng.standard_normal(inst.Ap[1])
        db = rng.standard_normal(m)
        for dA, dbb in ((dAx, 0 * db), (0 * dAx, db)):
            fd = (loss(_solve(inst, inst.Ax + eps * dA, inst.b + eps * dbb)) -
                  loss(_solve(inst, inst.Ax - eps * dA, inst.b - eps * dbb))) / (2 * eps)
            an = gAx @ dA + gb @ dbb
            assert abs(fd - an) <= 2e-2 * max(abs(an), 1.0), (fd, an)


def test_gradient_wrt_C_values_is_Z():
    """dL/dC stored values = Z_ij (diagonal) or 2 Z_ij (off-diagonal)."""
    inst = instances.maxcut(12, 0.4, seed=2)
    r0 = _solve(inst, inst.Ax.copy(), inst.b.copy())
    rng = np.random.default_rng(0)
    G = rng.standard_normal((12, 12))
    G = G + G.T
    gb, Z, gAx = adjoint_ref.vjp(inst, r0["y"], r0["X"], np.zeros(inst.m), G)
    from oracle import kernels_ref as K
    i, j = K.packed_to_ij(12, inst.Ai[:inst.Ap[1]])
    np.testing.assert_allclose(gAx[:inst.Ap[1]], np.where(i == j, 1, 2) * Z[i, j])
    np.testing.assert_allclose(Z, Z.T)
