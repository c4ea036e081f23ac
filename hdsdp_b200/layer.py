"""Differentiable SDP layer: torch.autograd.Function over the C ABI.

Forward solves a problem of one dense SDP block (data given as the reference's CSC layout:
column 0 is C, columns 1..m the A_i, packed lower-triangle rows) through
HDSDPOptimize and returns (y*, X*). Backward calls HDSDPAdjoint, which
differentiates the optimality conditions at the final iterate on the GPU and
returns the gradients with respect to the CSC values and b. This is a thin
ctypes shim: all arithmetic runs in libhdsdp_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .api import Solver, _dp


class SDPLayer(torch.autograd.Function):
    """y, X = SDPLayer.apply(Ax, b, Ap, Ai, n) with Ax (values) and b differentiable (FP64)."""

    @staticmethod
    def forward(ctx, Ax, b, Ap, Ai, n):
        m = len(Ap) - 2  # CSC column pointer of columns 0 (C) .. m (A_m)
        ax = np.ascontiguousarray(Ax.detach().cpu().numpy(), dtype=np.float64)
        bv = np.ascontiguousarray(b.detach().cpu().numpy(), dtype=np.float64)
        s = Solver()
        s.init(m, 1)
        if s.set_cone(m, n, Ap, Ai, ax) != 0:
            s.close()
            raise RuntimeError("HDSDPSetCone rejected the block")
        s.set_dual_objective(bv)
        s.set_primal_refinement(False)
        s.optimize(0)
        _, _, y = s.get_row_dual()
        X, _ = s.get_cone_values()
        ctx.solver = s          # keeps the device factors (and the CSC arrays) for the backward pass
        ctx.n, ctx.m, ctx.nnz = n, m, ax.size
        ctx.status = s.status()
        return torch.from_numpy(y), torch.from_numpy(np.ascontiguousarray(X))

    @staticmethod
    def backward(ctx, gy, gX):
        L = _lib.load()
        s = ctx.solver
        n, m = ctx.n, ctx.m
        gyv = np.ascontiguousarray((gy if gy is not None else torch.zeros(m)).detach().cpu().numpy(),
                                   dtype=np.float64)
        GX = np.zeros((n, n)) if gX is None else gX.detach().cpu().numpy().astype(np.float64)
        GX = np.asfortranarray(0.5 * (GX + GX.T))
        gb = np.zeros(m)
        gC = np.zeros((n, n), order="F")
        gAx = np.zeros(ctx.nnz)
        r = L.HDSDPAdjoint(s.h, _dp(gyv), _dp(GX), _dp(gb), _dp(gC), _dp(gAx))
        if r != 0:
            raise RuntimeError("HDSDPAdjoint failed (%d)" % r)
        return torch.from_numpy(gAx), torch.from_numpy(gb), None, None, None


def solve_layer(Ax, b, Ap, Ai, n):
    return SDPLayer.apply(Ax, b, Ap, Ai, n)
