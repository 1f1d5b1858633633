"""Autograd Functions of the projector path, API-compatible with
``xrecon.projector.functions`` (XRecon xrecon/projector/functions.py:96-302).

Each Function's backward is the partner transpose operator, exactly as in the
reference: Projection <-> ProjectionTranspose, BackProjection <->
BackProjectionTranspose, WeightedBackProjection <-> its transpose.  Only the
options/angles are saved (no activations).  ``option`` may be the packed
options tensor (reference calling convention) or a
:class:`~xrecon_b200.backend.HostGeometry`.
"""
from __future__ import annotations

import torch
from torch.autograd import Function

from . import backend as _B


def _c(t):
    return t if t.is_contiguous() else t.contiguous()


def _make(name: str, fwd, bwd):
    def forward(ctx, input, option, angles):
        out = fwd(_c(input), option, angles)
        ctx.option = option
        ctx.save_for_backward(angles)
        return out

    def backward(ctx, grad_output):
        (angles,) = ctx.saved_tensors
        return bwd(_c(grad_output), ctx.option, angles), None, None

    return type(name, (Function,), {"forward": staticmethod(forward), "backward": staticmethod(backward)})


Projection2d = _make("Projection2d", _B.forward_projection2d, _B.projection_transpose2d)
ProjectionTranspose2d = _make("ProjectionTranspose2d", _B.projection_transpose2d, _B.forward_projection2d)
BackProjection2d = _make("BackProjection2d", _B.backward_projection2d, _B.backward_projection_transpose2d)
BackProjectionTranspose2d = _make("BackProjectionTranspose2d", _B.backward_projection_transpose2d,
                                  _B.backward_projection2d)
WeightedBackProjection2d = _make("WeightedBackProjection2d", _B.weighted_backward_projection2d,
                                 _B.weighted_backward_projection_transpose2d)
WeightedBackProjectionTranspose2d = _make("WeightedBackProjectionTranspose2d",
                                          _B.weighted_backward_projection_transpose2d,
                                          _B.weighted_backward_projection2d)

Projection3d = _make("Projection3d", _B.forward_projection3d, _B.projection_transpose3d)
ProjectionTranspose3d = _make("ProjectionTranspose3d", _B.projection_transpose3d, _B.forward_projection3d)
BackProjection3d = _make("BackProjection3d", _B.backward_projection3d, _B.backward_projection_transpose3d)
BackProjectionTranspose3d = _make("BackProjectionTranspose3d", _B.backward_projection_transpose3d,
                                  _B.backward_projection3d)
WeightedBackProjection3d = _make("WeightedBackProjection3d", _B.weighted_backward_projection3d,
                                 _B.weighted_backward_projection_transpose3d)
WeightedBackProjectionTranspose3d = _make("WeightedBackProjectionTranspose3d",
                                          _B.weighted_backward_projection_transpose3d,
                                          _B.weighted_backward_projection3d)


def _make_helical(name: str, fwd, bwd):
    """Helical Functions (functions.py:305-388 of the reference): the same
    pairing, with ``source_pos`` [4, V] as a fourth, non-differentiable input."""
    def forward(ctx, input, option, angles, source_pos):
        out = fwd(_c(input), option, angles, source_pos)
        ctx.option = option
        ctx.save_for_backward(angles, source_pos)
        return out

    def backward(ctx, grad_output):
        angles, source_pos = ctx.saved_tensors
        return bwd(_c(grad_output), ctx.option, angles, source_pos), None, None, None

    return type(name, (Function,), {"forward": staticmethod(forward), "backward": staticmethod(backward)})


ProjectionHelical3d = _make_helical("ProjectionHelical3d", _B.forward_projection_helical3d,
                                    _B.projection_transpose_helical3d)
ProjectionTransposeHelical3d = _make_helical("ProjectionTransposeHelical3d", _B.projection_transpose_helical3d,
                                             _B.forward_projection_helical3d)
BackProjectionHelical3d = _make_helical("BackProjectionHelical3d", _B.backward_projection_helical3d,
                                        _B.backward_projection_transpose_helical3d)
BackProjectionTransposeHelical3d = _make_helical("BackProjectionTransposeHelical3d",
                                                 _B.backward_projection_transpose_helical3d,
                                                 _B.backward_projection_helical3d)
WeightedBackProjectionHelical3d = _make_helical("WeightedBackProjectionHelical3d",
                                                _B.weighted_backward_projection_helical3d,
                                                _B.weighted_backward_projection_transpose_helical3d)
WeightedBackProjectionTransposeHelical3d = _make_helical("WeightedBackProjectionTransposeHelical3d",
                                                         _B.weighted_backward_projection_transpose_helical3d,
                                                         _B.weighted_backward_projection_helical3d)


class ProjectionLeastSquares(Function):
    """``0.5 * ||A x - y||^2`` summed over the batch, with A the projection
    (2D or 3D by the rank of ``x``), evaluated over chunks of views.

    Forward projects one chunk of ``view_chunk`` views at a time and keeps
    only the scalar; backward recomputes each chunk's residual
    ``r_c = A_c x - y_c`` and accumulates ``A_c^T r_c``, the hand-written
    transpose that is the backward of ``Projection2d/3d``.  Nothing of
    sinogram size is saved between forward and backward, and at most one
    chunk's sinogram is alive, so batched 3D gradients need
    O(volume + view_chunk * detector) memory instead of O(views * detector).
    Sums are accumulated in FP64.

    ``y`` is not differentiated (the measured data).
    """

    @staticmethod
    def forward(ctx, x, y, option, angles, view_chunk: int):
        dim = x.dim() - 2
        fwd = _B.forward_projection2d if dim == 2 else _B.forward_projection3d
        xc = _c(x)
        V = angles.numel()
        total = torch.zeros((), dtype=torch.float64, device=x.device)
        for v0 in range(0, V, view_chunk):
            v1 = min(V, v0 + view_chunk)
            r = fwd(xc, option, angles[v0:v1].contiguous()) - y[:, :, v0:v1]
            total += r.double().square().sum()
        ctx.option = option
        ctx.view_chunk = view_chunk
        ctx.save_for_backward(x, y, angles)
        return (0.5 * total).to(x.dtype)

    @staticmethod
    def backward(ctx, grad_output):
        x, y, angles = ctx.saved_tensors
        dim = x.dim() - 2
        fwd = _B.forward_projection2d if dim == 2 else _B.forward_projection3d
        adj = _B.projection_transpose2d if dim == 2 else _B.projection_transpose3d
        xc = _c(x)
        V = angles.numel()
        grad = torch.zeros_like(x)  # also the gradient of a scan with no views
        for v0 in range(0, V, ctx.view_chunk):
            v1 = min(V, v0 + ctx.view_chunk)
            a = angles[v0:v1].contiguous()
            r = fwd(xc, ctx.option, a) - y[:, :, v0:v1]
            grad.add_(adj(_c(r), ctx.option, a))
        return grad * grad_output, None, None, None, None


def projection_least_squares(x, y, option, angles, view_chunk: int = 32):
    """Differentiable ``0.5 * ||A x - y||^2`` with view-chunked recomputation
    (see :class:`ProjectionLeastSquares`)."""
    if view_chunk < 1:
        raise ValueError("view_chunk must be >= 1")
    return ProjectionLeastSquares.apply(x, y, option, angles, int(view_chunk))
