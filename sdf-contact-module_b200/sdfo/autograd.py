"""torch.autograd front end of the query kernels.

``sdf_query(grid, points, payload=None, mode=...)`` returns ``(gap, grad)``
and is differentiable w.r.t. ``points`` (dL/dp = dgap * grad + H dgrad with
the interpolant's Hessian H) and, when ``payload`` is given, w.r.t. the grid's
stored {phi, n} values.  Forward and backward are the hand-written kernels
(sdfo_query / sdfo_query_backward); there is no reference counterpart (the
reference has no autodiff).
"""
from __future__ import annotations

import torch

from . import _native as N


class SDFQuery(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, payload, grid, mode):
        g = grid if payload is None else grid.view(payload)
        out = g.query_tensors(points, mode=mode, valid=False)
        ctx.grid = g
        ctx.mode = mode
        ctx.save_for_backward(points)
        return out["gap"], out["grad"]

    @staticmethod
    def backward(ctx, dgap, dgrad):
        (points,) = ctx.saved_tensors
        g = ctx.grid
        need_p = ctx.needs_input_grad[0]
        need_v = ctx.needs_input_grad[1]
        dgrid = None
        if need_v:
            dgrid = torch.zeros((g.stored_voxels, 4), dtype=torch.float32, device=points.device)
        pts32 = points.detach().to(torch.float32).contiguous()
        dpts = g.query_backward(pts32, dgap, dgrad, mode=ctx.mode, dgrid=dgrid,
                                want_points=need_p)
        if dpts is not None and points.dtype != torch.float32:
            dpts = dpts.to(points.dtype)
        return dpts, dgrid, None, None


def sdf_query(grid, points, payload=None, mode=N.TRICUBIC):
    """Differentiable Trilinear/Tricubic query: returns (gap (N,), grad (N,3))."""
    m = N.mode_id(mode)
    if m not in (N.TRILINEAR, N.TRICUBIC):
        raise ValueError("sdf_query is differentiable for Trilinear and Tricubic")
    return SDFQuery.apply(points, payload, grid, m)
