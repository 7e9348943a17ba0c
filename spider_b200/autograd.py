"""PJ 3Q as a differentiable operator.

``PJ3Q`` is a ``torch.autograd.Function``: forward is the trilinear
projection of ``spi_pj3q`` (WPRO_N, wpro_n.f:44-150), backward is its exact
adjoint ``spi_pj3q_adjoint`` -- the trilinear insertion that spreads each
projection value back onto the 8 voxels around the same sample position.  The
backward recomputes the rotated sample positions from the angles instead of
storing them, so the autograd graph holds only the angles.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ops


class PJ3Q(torch.autograd.Function):
    @staticmethod
    def forward(fctx, vol: torch.Tensor, angles: np.ndarray, ri: float, lib_ctx):
        if not vol.is_cuda:
            raise ops.SpiderError(101, "PJ3Q needs a CUDA volume (there is no CPU path)")
        fctx.angles = angles
        fctx.ri = ri
        fctx.lib_ctx = lib_ctx
        fctx.shape = tuple(vol.shape)
        return ops.pj3q(vol.detach().contiguous().float(), angles, ri, ctx=lib_ctx)

    @staticmethod
    def backward(fctx, grad: torch.Tensor):
        g = ops.pj3q_adjoint(grad.detach().contiguous().float(), fctx.angles, fctx.shape, fctx.ri,
                             ctx=fctx.lib_ctx)
        return g, None, None, None


def pj3q(vol: torch.Tensor, angles, ri: float | None = None, ctx: ops.Context | None = None) -> torch.Tensor:
    """Differentiable ``PJ 3Q`` of a CUDA volume [nz, ny, nx] -> [nang, ny, nx]."""
    if ri is None:
        ri = float(min(vol.shape) // 2 - 2)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    return PJ3Q.apply(vol, ang, float(ri), ctx or ops.default_context(vol.device.index or 0))
