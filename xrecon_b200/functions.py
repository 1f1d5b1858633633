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
