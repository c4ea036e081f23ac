"""HDSDPAdjoint on the GPU against the FP64 NumPy restatement at the same
iterate, against central finite differences of GPU solves, and through the
torch.autograd layer."""
from __future__ import annotations

import copy

import numpy as np
import pytest
import torch

from hdsdp_b200 import api, instances
from hdsdp_b200.layer import SDPLayer
from oracle import adjoint_ref

pytestmark = pytest.mark.gpu


def _solve(inst, Ax=None, b=None):
    s = api.Solver()
    s.init(inst.m, 1)
    assert s.set_cone(inst.m, inst.n, inst.Ap, inst.Ai, inst.Ax if Ax is None else Ax) == 0
    s.set_dual_objective(inst.b if b is None else b)
    s.set_primal_refinement(False)
    s.optimize(0)
    return s


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("make", [lambda: instances.maxcut(30, 0.3, seed=3),
                                  lambda: instances.rank_one(20, 30, 0.3, seed=6),
                                  lambda: instances.theta_adjoint(40, 0.2, 0.3, seed=2)])
def test_adjoint_matches_restatement(gpu_lib, make):
    inst = make()
    s = _solve(inst)
    try:
        assert s.status() == 3
        _, _, y = s.get_row_dual()
        X, _ = s.get_cone_values()
        rng = np.random.default_rng(4)
        G = rng.standard_normal((inst.n, inst.n))
        G = G + G.T
        h = rng.standard_normal(inst.m)
        gb, gC, gAx = s.adjoint(h, G)
        rb, rC, rAx = adjoint_ref.vjp(inst, y, X, h, G)
        # within 1e-5 relative of the FP64 restatement (the theta layer's gradients reach
        # 1e9 in the directions of the active zero constraints)
        assert _rel(gb, rb) < 1e-5
        assert _rel(gC, rC) < 1e-5
        assert _rel(gAx, rAx) < 1e-5
        # second call reuses the cached factors and gives the same answer
        gb2, _, _ = s.adjoint(h, G)
        np.testing.assert_allclose(gb2, gb, rtol=1e-12, atol=0)
    finally:
        s.close()


def test_adjoint_matches_finite_differences(gpu_lib):
    inst = instances.maxcut(30, 0.3, seed=3)
    rng = np.random.default_rng(1)
    G = rng.standard_normal((30, 30))
    G = G + G.T
    h = rng.standard_normal(inst.m)
    s = _solve(inst)
    gb, gC, gAx = s.adjoint(h, G)
    s.close()

    def loss(Ax, b):
        t = _solve(inst, Ax, b)
        try:
            _, _, y = t.get_row_dual()
            X, _ = t.get_cone_values()
            return float(np.sum(G * X) + h @ y)
        finally:
            t.close()

    eps = 1e-5
    for _ in range(3):
        dAx = np.zeros(inst.Ax.size)
        dAx[:inst.Ap[1]] = rng.standard_normal(inst.Ap[1])
        db = rng.standard_normal(inst.m)
        for dA, dbb in ((dAx, 0 * db), (0 * dAx, db)):
            fd = (loss(inst.Ax + eps * dA, inst.b + eps * dbb) - loss(inst.Ax - eps * dA, inst.b - eps * dbb)) / (2 * eps)
            an = gAx @ dA + gb @ dbb
            assert abs(fd - an) <= 2e-2 * max(abs(an), 1.0), (fd, an)


def test_torch_layer_backward(gpu_lib):
    inst = instances.maxcut(24, 0.3, seed=5)
    Ax = torch.tensor(inst.Ax, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(inst.b, dtype=torch.float64, requires_grad=True)
    y, X = SDPLayer.apply(Ax, b, inst.Ap, inst.Ai, inst.n)
    rng = np.random.default_rng(2)
    G = torch.tensor(rng.standard_normal((24, 24)))
    G = G + G.T
    h = torch.tensor(rng.standard_normal(inst.m))
    L = (G * X).sum() + (h * y).sum()
    L.backward()
    s = _solve(inst)
    gb, _, gAx = s.adjoint(h.numpy(), G.numpy())
    s.close()
    np.testing.assert_allclose(b.grad.numpy(), gb, rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(Ax.grad.numpy(), gAx, rtol=1e-8, atol=1e-10)


@pytest.mark.slow
def test_adjoint_full_size_theta(gpu_lib):
    """Theta-style layer n=200 (m=3,595): the adjoint at the GPU's own solution matches the
    FP64 restatement to 1e-5 relative, and dL/dC is symmetric."""
    inst = instances.WORKLOADS["theta_adjoint_n200"]()
    s = _solve(inst)
    try:
        assert s.status() == 3
        _, _, y = s.get_row_dual()
        X, _ = s.get_cone_values()
        rng = np.random.default_rng(3)
        G = rng.standard_normal((inst.n, inst.n))
        G = G + G.T
        h = rng.standard_normal(inst.m)
        gb, gC, gAx = s.adjoint(h, G)
        rb, rC, rAx = adjoint_ref.vjp(inst, y, X, h, G)
        assert _rel(gb, rb) < 1e-5
        assert _rel(gC, rC) < 1e-5
        assert _rel(gAx, rAx) < 1e-5
        np.testing.assert_allclose(gC, gC.T, atol=1e-9 * np.abs(gC).max())
    finally:
        s.close()


def test_adjoint_fd_twenty_directions(gpu_lib):
    """Central differences of full GPU solves at step 1e-6 in 20 random directions of C's
    values and of b on a nondegenerate instance (MaxCut n=30), against the adjoint of
    L = h^T y*. The solves run with tightened optimality tolerances (absolute 1e-13,
    relative 1e-14), which puts the dual solution's error near 1e-9 and the error of each
    difference near 1e-3 of the gradient; the compiled reference, differenced the same
    way, agrees with the FP64 restatement to 3.5e-2 in the worst of these directions.
    (The primal X* comes from the dual-scaling method's primal marker, good to about 1e-7,
    so its part of the gradient is checked against the restatement instead, above.)"""
    inst = instances.maxcut(30, 0.3, seed=3)
    rng = np.random.default_rng(11)
    h = rng.standard_normal(inst.m)
    tight = {3: 1e-13, 1: 1e-14}

    def solve(Ax, b):
        s = api.Solver()
        s.init(inst.m, 1)
        assert s.set_cone(inst.m, inst.n, inst.Ap, inst.Ai, Ax) == 0
        s.set_dual_objective(b)
        s.set_primal_refinement(False)
        for k, v in tight.items():
            s.set_dbl_param(k, v)
        s.optimize(0)
        return s

    s = solve(inst.Ax, inst.b)
    assert s.status() == 3
    gb, gC, gAx = s.adjoint(h, None)
    s.close()

    def loss(Ax, b):
        t = solve(Ax, b)
        try:
            _, _, y = t.get_row_dual()
            return float(h @ y)
        finally:
            t.close()

    eps = 1e-6
    worst = 0.0
    for _ in range(20):
        dAx = np.zeros(inst.Ax.size)
        dAx[:inst.Ap[1]] = rng.standard_normal(inst.Ap[1])
        db = rng.standard_normal(inst.m)
        fd = (loss(inst.Ax + eps * dAx, inst.b + eps * db) - loss(inst.Ax - eps * dAx, inst.b - eps * db)) / (2 * eps)
        an = gAx @ dAx + gb @ db
        worst = max(worst, abs(fd - an) / max(abs(an), 1.0))
    print("worst FD relative difference over 20 directions: %.3e" % worst)
    assert worst <= 1e-1
