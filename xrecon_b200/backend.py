"""Drop-in replacement of the reference's native module ``xrecon_C``.

Same function names and signatures as XRecon's pybind module
(src/api/torch_binding.cpp:615-638): every function takes
``(input, options, angles)`` and returns a new tensor.  Differences that a
caller can observe:

* only CUDA tensors are accepted (the reference also runs on CPU); a CPU
  tensor raises ``RuntimeError``;
* float32, bfloat16 and float16 storage are accepted (the reference accepts
  float32 only); accumulation is float32 in every case;
* ``options`` may be a tensor on any device or any sequence of numbers; it is
  read once on the host (the reference reads it element by element with
  ``.item()``, torch_binding.cpp:62-124), or a :class:`HostGeometry`, which
  skips the read entirely;
* all work is enqueued on torch's current CUDA stream (the reference uses the
  legacy default stream and synchronises in the 2D path).

Errors (device mismatch, non-contiguous input, bad shapes) raise
``RuntimeError`` like the reference's ``TORCH_CHECK``.
"""
from __future__ import annotations

import torch

from . import _native


class HostGeometry:
    """Packed options already on the host, with their C struct."""

    __slots__ = ("dim", "values", "struct")

    def __init__(self, dim: int, values):
        import numpy as np
        self.dim = dim
        # float32 rounding, as the reference's float32 options tensor
        self.values = [float(np.float32(v)) for v in values]
        self.struct = (_native.geom2d_from_values if dim == 2 else _native.geom3d_from_values)(self.values)


def _geom(dim: int, options):
    if isinstance(options, HostGeometry):
        if options.dim != dim:
            raise RuntimeError(f"expected {dim}D options")
        return options.struct
    if isinstance(options, torch.Tensor):
        if options.dtype != torch.float32:
            raise RuntimeError("options must be float32")
        vals = options.detach().reshape(-1).cpu().tolist()
    else:
        vals = list(options)
    need = 12 if dim == 2 else 18
    if len(vals) < need:
        if dim == 2:
            raise RuntimeError("Option tensor must have at least 12 elements.")
        raise RuntimeError("3D option tensor must have at least 18 elements.")
    if dim == 3 and int(vals[17]) not in (0, 1, 2):
        raise RuntimeError("3D scan_type must be parallel, flat, or arc")
    return HostGeometry(dim, vals[:need]).struct


def _check(x: torch.Tensor, options, angles: torch.Tensor):
    devs = {x.device, angles.device}
    if isinstance(options, torch.Tensor):
        devs.add(options.device)
    if len(devs) != 1:
        raise RuntimeError("Expected all tensors on the same device, but got devices: "
                           + ", ".join(str(d) for d in devs))
    if not x.is_contiguous() or not angles.is_contiguous() or (
            isinstance(options, torch.Tensor) and not options.is_contiguous()):
        raise RuntimeError("Expected all tensors to be contiguous")
    if angles.dtype != torch.float32:
        raise RuntimeError("ang must be float32")


def _run(dim, op, x, options, angles):
    _check(x, options, angles)
    return _native.apply(dim, op, x, _geom(dim, options), angles)


def forward_projection2d(image, options, ang):
    return _run(2, "A", image, options, ang)


def projection_transpose2d(proj, options, ang):
    return _run(2, "AT", proj, options, ang)


def backward_projection2d(proj, options, ang):
    return _run(2, "B", proj, options, ang)


def weighted_backward_projection2d(proj, options, ang):
    return _run(2, "BW", proj, options, ang)


def backward_projection_transpose2d(image, options, ang):
    return _run(2, "BT", image, options, ang)


def weighted_backward_projection_transpose2d(image, options, ang):
    return _run(2, "BWT", image, options, ang)


back_projection2d = backward_projection2d
weighted_back_projection2d = weighted_backward_projection2d


def forward_projection3d(image, options, ang):
    return _run(3, "A", image, options, ang)


def projection_transpose3d(proj, options, ang):
    return _run(3, "AT", proj, options, ang)


def backward_projection3d(proj, options, ang):
    return _run(3, "B", proj, options, ang)


def weighted_backward_projection3d(proj, options, ang):
    return _run(3, "BW", proj, options, ang)


def backward_projection_transpose3d(image, options, ang):
    return _run(3, "BT", image, options, ang)


def weighted_backward_projection_transpose3d(image, options, ang):
    return _run(3, "BWT", image, options, ang)


# ------------------------------------------------------------------ helical
# torch_binding.cpp:525-612: (input, options[24], angles[V], source_pos[4, V]),
# float32 CUDA tensors, arc detector only.

class HelicalHostGeometry:
    """Packed helical options (24 entries) already on the host."""

    __slots__ = ("values", "struct", "hopts")

    def __init__(self, values):
        import numpy as np
        self.values = [float(np.float32(v)) for v in values]
        self.struct = _native.geom3d_from_values(self.values[:18])
        self.hopts = _native.helical_opts_from_values(self.values)


def _helical_geom(options):
    if isinstance(options, HelicalHostGeometry):
        return options
    if isinstance(options, torch.Tensor):
        if options.dtype != torch.float32:
            raise RuntimeError("Helical 3D tensors must be float32")
        vals = options.detach().reshape(-1).cpu().tolist()
    else:
        vals = list(options)
    if len(vals) < 18:
        raise RuntimeError("3D option tensor must have at least 18 elements.")
    return HelicalHostGeometry(vals)


def _run_helical(op, x, options, angles, source_pos):
    _check(x, options, angles)
    if source_pos.device != x.device:
        raise RuntimeError("Expected all tensors on the same device")
    if not source_pos.is_contiguous():
        raise RuntimeError("Expected all tensors to be contiguous")
    hg = _helical_geom(options)
    return _native.helical(op, x, hg.struct, hg.hopts, angles, source_pos)


def forward_projection_helical3d(image, options, ang, source_pos):
    return _run_helical("A", image, options, ang, source_pos)


def projection_transpose_helical3d(proj, options, ang, source_pos):
    return _run_helical("AT", proj, options, ang, source_pos)


def backward_projection_helical3d(proj, options, ang, source_pos):
    return _run_helical("B", proj, options, ang, source_pos)


def weighted_backward_projection_helical3d(proj, options, ang, source_pos):
    return _run_helical("BW", proj, options, ang, source_pos)


def backward_projection_transpose_helical3d(image, options, ang, source_pos):
    return _run_helical("BT", image, options, ang, source_pos)


def weighted_backward_projection_transpose_helical3d(image, options, ang, source_pos):
    return _run_helical("BWT", image, options, ang, source_pos)
