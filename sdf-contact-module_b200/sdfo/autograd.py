"""torch.autograd front end of the query kernels.

``sdf_query(grid, points, payload=None, mode=...)`` returns ``(gap, grad)``
and is differentiable w.r.t. ``points`` (dL/dp = dgap * grad + H dgrad with
the interpolant's Hessian H) and, when ``payload`` is given, w.r.t. the grid's
stored {phi, n} values.  There is no reference counterpart (the reference has
no autodiff).

Float32 points take the saved-linearisation path: the forward kernel
(sdfo_query_linearize) also writes the per-point symmetric Hessian, and the
backward kernel (sdfo_query_backward_saved) is then elementwise for dL/dp
and needs only the corner weights (not the grid values) for dL/dgrid, so the
grid stencil is gathered once per forward+backward.  Float64 points use the
plain FP64-indexed forward and the stencil-regathering backward
(sdfo_query_backward).
"""
from __future__ import annotations

import torch

from . import _native as N


class SDFQuery(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, payload, grid, mode):
        g = grid if payload is None else grid.view(payload)
        ctx.grid = g
        ctx.mode = mode
        ctx.saved = None
        if points.dtype == torch.float32 and points.is_cuda:
            pts = points.detach().contiguous().reshape(-1, 3)
            if ctx.needs_input_grad[0]:
                out = g.query_linearize(pts, mode=mode)
                ctx.saved = out
            else:
                out = g.query_tensors(pts, mode=mode, valid=True)
                ctx.saved = dict(valid=out["valid"])
            ctx.save_for_backward(points)
            return out["gap"], out["grad"]
        out = g.query_tensors(points, mode=mode, valid=False)
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
        pts32 = points.detach().to(torch.float32).contiguous().reshape(-1, 3)
        if ctx.saved is not None:
            dpts = g.query_backward_saved(pts32, ctx.saved, dgap, dgrad, mode=ctx.mode,
                                          dgrid=dgrid, want_points=need_p)
        else:
            dpts = g.query_backward(pts32, dgap, dgrad, mode=ctx.mode, dgrid=dgrid,
                                    want_points=need_p)
        if dpts is not None:
            dpts = dpts.reshape(points.shape)
            if points.dtype != torch.float32:
                dpts = dpts.to(points.dtype)
        return dpts, dgrid, None, None


def sdf_query(grid, points, payload=None, mode=N.TRICUBIC):
    """Differentiable Trilinear/Tricubic query: returns (gap (N,), grad (N,3))."""
    m = N.mode_id(mode)
    if m not in (N.TRILINEAR, N.TRICUBIC):
        raise ValueError("sdf_query is differentiable for Trilinear and Tricubic")
    return SDFQuery.apply(points, payload, grid, m)
