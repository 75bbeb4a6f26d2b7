"""``torch.autograd.Function`` around the MSGB forward and its exact transpose.

The forward stores only the frozen beam selection (flat indices and c_pos
values); the backward recomputes every Gaussian inside the transpose kernels
(no per-(beam, time, sensor) state is kept).
"""

from __future__ import annotations

import torch


class MSGBForward(torch.autograd.Function):
    """``y = A p0``; ``backward`` returns ``A^T grad_y`` with the selection frozen."""

    @staticmethod
    def forward(ctx, p0, solver, domain, sensors, ts, wpt, selection=None):
        if selection is None:
            data = solver.forward(p0, domain, sensors, ts, wpt)
            selection = solver.last_selection
        else:
            data = solver.forward_frozen(p0, domain, sensors, ts, wpt, selection)
        ctx.solver, ctx.domain, ctx.sensors, ctx.ts, ctx.wpt = solver, domain, sensors, ts, wpt
        ctx.selection = selection
        ctx.out_dtype = p0.dtype
        return data

    @staticmethod
    def backward(ctx, grad_out):
        img = ctx.solver.adjoint(grad_out.contiguous(), ctx.domain, ctx.sensors, ctx.ts, ctx.wpt,
                                 selection=ctx.selection)
        return img.to(ctx.out_dtype), None, None, None, None, None, None


def msgb_forward(p0, solver, domain, sensors, ts, wpt, selection=None):
    """Differentiable MSGB forward of a CUDA tensor ``p0``.  Without
    ``selection`` the beams are re-selected from p0 at every call, as
    ``MSGBSolver.forward`` does; with one, the selection stays frozen and the
    map is linear in p0."""
    return MSGBForward.apply(p0, solver, domain, sensors, ts, wpt, selection)
