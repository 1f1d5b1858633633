"""``Projector2d`` / ``Projector3d``: drop-in replacements of XRecon's
projector modules (xrecon/projector/projector.py:21-316 and
xrecon/projector/projector3d.py:29-287) running on the B200 kernels.

Same constructor arguments, buffers (``options``, ``weight``, ``filter``,
registered non-persistent unless ``trainable``), method names, shapes,
assertions and FBP/FDK semantics.  ``filtered_backprojection`` runs the fused
cosine-weight x Parker x filter kernel followed by the weighted backprojection
when no gradient is needed; when the sinogram, ``weight`` or ``filter``
require gradients it runs differentiable torch ops for the weighting and
filtering (FP32, TF32 disabled) followed by the weighted-backprojection
autograd Function.
"""
from __future__ import annotations

import math
from typing import List, Optional, Tuple, Union

import torch
import torch.nn as nn
from torch import Tensor

from . import _native
from .backend import HostGeometry
from .filters import filter_generate
from .backend import HelicalHostGeometry
from .functions import (
    BackProjection2d, BackProjection3d, BackProjectionHelical3d, BackProjectionTranspose2d,
    BackProjectionTranspose3d, BackProjectionTransposeHelical3d, Projection2d, Projection3d,
    ProjectionHelical3d, ProjectionTranspose2d, ProjectionTranspose3d, ProjectionTransposeHelical3d,
    WeightedBackProjection2d, WeightedBackProjection3d, WeightedBackProjectionHelical3d,
    WeightedBackProjectionTranspose2d, WeightedBackProjectionTranspose3d,
    WeightedBackProjectionTransposeHelical3d,
)
from .geometry import (
    ConeBeam3d, Detector3d, FanBeam2d, HelicalConeBeam3d, ParallelBeam2d, ParallelBeam3d, Volume2d, Volume3d,
    make_geometry2d, make_geometry3d, pack_options2d, pack_options3d,
)

_SCAN_ALIASES = {"para": "parallel", "parallel": "parallel", "flat": "flat", "arc": "arc"}


def mean_angle_step(angles: Tensor) -> Tensor:
    """Mean wrapped angular step |((d + pi) mod 2pi) - pi| (projector.py:303-313)."""
    if angles.numel() < 2:
        return angles.new_tensor(0.0)
    d = torch.diff(angles)
    return ((d + math.pi) % (2 * math.pi) - math.pi).abs().mean()


def parker_weights(angles: Tensor, gamma: Tensor, num_det: int) -> Tensor:
    """Short-scan weights (projector.py:208-246): sin^2 ramps of width
    2*(overscan - gamma) at the start and end of the scan, where
    overscan = max((range - pi)/2, gamma_max); ones for full scans."""
    V = angles.numel()
    ones = torch.ones((V, num_det), device=angles.device, dtype=angles.dtype)
    if V < 2:
        return ones
    beta = angles - angles[0]
    scan_range = beta[-1].abs()
    gamma_max = gamma.abs().max()
    if scan_range >= (2 * math.pi - 1e-4):
        return ones
    if scan_range < math.pi + 2.0 * gamma_max - mean_angle_step(angles):
        raise ValueError("Parker weighting requires a short-scan range of at least "
                         f"pi + 2 * gamma_max, got {scan_range.item():.6f} rad")
    overscan = torch.clamp((scan_range - math.pi) / 2.0, min=gamma_max)
    eps = torch.finfo(angles.dtype).eps
    left = 2.0 * (overscan - gamma)
    right = scan_range - 2.0 * (overscan + gamma)
    b = beta[:, None]
    w_left = torch.sin(0.5 * math.pi * b / torch.clamp(left, min=eps)[None, :]).pow(2)
    w_right = torch.sin(0.5 * math.pi * (scan_range - b) / torch.clamp(scan_range - right, min=eps)[None, :]).pow(2)
    w = torch.where(b < left[None, :], w_left, ones)
    w = torch.where(b > right[None, :], w_right, w)
    return w.clamp_(0.0, 1.0)


class _FilterRows(torch.autograd.Function):
    """Differentiable FBP pre-filter: ``out = corr_u(s * weight * parker, filt)``
    with the fused kernel, in FP32 without TF32.

    The adjoint of the correlation with ``filt`` is the correlation with the
    reversed filter, so the sinogram gradient runs through the same kernel;
    the (rarely trained) weight and filter gradients are reduced in FP64.
    """

    @staticmethod
    def forward(ctx, s, weight, filt, parker, nview, rows_per_view):
        Nu = s.shape[-1]
        sc = s.contiguous()
        out = _native.fbp_filter(sc, nview=nview, rows_per_view=rows_per_view,
                                 cosw=weight.detach().reshape(-1), filt=filt.detach().reshape(-1),
                                 parker=None if parker is None else parker.detach().reshape(nview, Nu))
        ctx.save_for_backward(sc, weight, filt, parker)
        ctx.nview, ctx.rows_per_view = nview, rows_per_view
        return out

    @staticmethod
    def backward(ctx, g):
        s, weight, filt, parker = ctx.saved_tensors
        Nu = s.shape[-1]
        h = _native.fbp_filter(g.contiguous(), nview=ctx.nview, rows_per_view=ctx.rows_per_view, cosw=None,
                               filt=filt.detach().reshape(-1).flip(0), parker=None)
        w = weight.detach().to(h.dtype)
        pk = None if parker is None else parker.detach()  # broadcasts against the sinogram
        gs = gw = gf = None
        if ctx.needs_input_grad[0]:
            gs = h * w if pk is None else h * w * pk
        if ctx.needs_input_grad[1]:
            t = (h.double() * s.double()) if pk is None else (h.double() * s.double() * pk.double())
            gw = t.reshape(-1, Nu).sum(0).reshape(weight.shape).to(weight.dtype)
        if ctx.needs_input_grad[2]:
            # d out[i] / d filt[m] = sw[i + m - (Nu - 1)]
            sw = s.double() * w.double() if pk is None else s.double() * w.double() * pk.double()
            a = sw.reshape(-1, Nu)
            b = g.double().reshape(-1, Nu)
            n = 4 * Nu
            fa = torch.fft.rfft(a, n=n)
            fb = torch.fft.rfft(b, n=n)
            cc = torch.fft.irfft((fa * fb.conj()).sum(0), n=n)  # cc[k] = sum_i b[i] a[i + k]
            idx = torch.arange(2 * Nu - 1, device=cc.device) - (Nu - 1)
            gf = cc[idx % n].reshape(filt.shape).to(filt.dtype)
        return gs, gw, gf, None, None, None


class _ProjectorBase(nn.Module):
    _dim = 0

    def _host(self) -> HostGeometry:
        return self._host_geom

    @staticmethod
    def _prepare_angles(angles: Tensor, ref: Tensor) -> Tensor:
        return angles.to(device=ref.device, dtype=torch.float32 if ref.dtype in (torch.bfloat16, torch.float16)
                         else ref.dtype).contiguous()

    @staticmethod
    def _mean_angle_step(angles: Tensor) -> Tensor:
        return mean_angle_step(angles)

    def _fbp(self, sino: Tensor, angles: Tensor, filter, filter_type, redundant, parker: bool,
             rows_per_view: int) -> Tensor:
        self._check_sino_angles(sino, angles)
        if filter is not None:
            filt = filter
        elif filter_type is None or filter_type.lower() == self.filter_type:
            filt = self.filter
        else:
            filt = self._filter_generate(filter_type.lower(), dtype=torch.float32).to(sino.device)
        pw = None
        if parker:
            pw = self.parker_weight(angles)
            if redundant is None:
                redundant = False
        elif redundant is None:
            redundant = True
        scale = self._mean_angle_step(angles.to(torch.float32))
        if redundant:
            scale = scale / 2
        Nu = self._num_u()
        wt = self.weight
        needs_grad = torch.is_grad_enabled() and (
            sino.requires_grad or (isinstance(filt, Tensor) and filt.requires_grad) or wt.requires_grad)
        if needs_grad:
            pw_t = None if pw is None else pw.to(device=sino.device, dtype=torch.float32)
            filtered = _FilterRows.apply(sino.to(torch.float32), wt, filt, pw_t, angles.numel(), rows_per_view)
            recon = self.backprojection_weighted(filtered.contiguous(), angles)
            return recon * scale.to(device=recon.device, dtype=recon.dtype)
        with torch.no_grad():
            s = sino if sino.is_contiguous() else sino.contiguous()
            filtered = _native.fbp_filter(
                s, nview=angles.numel(), rows_per_view=rows_per_view,
                cosw=wt.detach().reshape(-1), filt=filt.detach().reshape(-1),
                parker=None if pw is None else pw.detach().reshape(angles.numel(), Nu))
            recon = self.backprojection_weighted(filtered, angles)
            if sino.dtype != torch.float32:
                recon = recon.to(sino.dtype)
            return recon * scale.to(device=recon.device, dtype=recon.dtype)


class Projector2d(_ProjectorBase):
    """Distance-driven 2D CT projector (parallel / fan-flat / fan-arc).

    Shapes: image [B, C, H, W], angles [V], sino [B, C, V, Nu].
    """
    _dim = 2

    def __init__(self, image_size: Union[int, Tuple[int, int], List[int], Volume2d],
                 num_det=None, pix_size=None, det_size: Optional[float] = None,
                 iso_source: float = 0.0, source_detector: float = 0.0, pixshift=0.0,
                 binshift: float = 0.0, scan_type: str = "flat", filter_type: str = "ramp",
                 trainable: bool = False, dtype=None) -> None:
        super().__init__()
        if isinstance(image_size, Volume2d):
            volume = image_size
            if isinstance(num_det, (FanBeam2d, ParallelBeam2d)) and pix_size is None:
                pix_size = num_det
            if not isinstance(pix_size, (FanBeam2d, ParallelBeam2d)):
                raise TypeError("When image_size is Volume2d, pix_size should be a 2D geometry object")
            geometry = pix_size
        else:
            if num_det is None or pix_size is None or det_size is None:
                raise TypeError("num_det, pix_size and det_size are required with the legacy constructor")
            volume = Volume2d(image_size, pix_size, pixshift)
            geometry = make_geometry2d(scan_type, num_det, det_size, iso_source, source_detector, binshift)
        scan = geometry.scan_type.lower().strip()
        scan = _SCAN_ALIASES.get(scan, scan)
        if scan not in ("parallel", "flat", "arc"):
            raise ValueError(f"Unsupported scan_type: {scan}")
        W, H = volume.size
        sx, sy = volume.spacing
        shx, shy = volume.shift
        self.image_size = (W, H)
        self.pix_size = (sx, sy)
        self.volume = volume
        self.geometry = geometry
        self.num_det = geometry.detector.count
        self.scan_type = scan
        self.filter_type = filter_type.lower().strip()
        self.iso_source = float(geometry.iso_source)
        self.source_detector = float(geometry.source_detector)
        self._default_dtype = dtype or torch.float32
        self.det_size = geometry.effective_det_spacing
        self.binshift = geometry.effective_det_shift
        self.pixshift = (shx * sx, shy * sy)
        packed = pack_options2d(volume, geometry)
        self._host_geom = HostGeometry(2, packed)
        self.register_buffer("options", torch.tensor(packed, dtype=self._default_dtype), persistent=False)
        w = self._make_cosine_weight(dtype=self._default_dtype)
        if trainable:
            self.weight = nn.Parameter(w.clone())
        else:
            self.register_buffer("weight", w, persistent=False)
        f = self._filter_generate(filter_type=self.filter_type, dtype=self._default_dtype)
        if trainable:
            self.filter = nn.Parameter(f.clone())
        else:
            self.register_buffer("filter", f, persistent=False)

    def _num_u(self) -> int:
        return self.num_det

    def forward(self, image: Tensor, angles: Tensor) -> Tensor:
        return self.projection(image, angles)

    def projection(self, image: Tensor, angles: Tensor) -> Tensor:
        _, _, h, w = image.shape
        assert (w, h) == self.image_size, f"Expected input image size {self.image_size[::-1]}, but got {(h, w)}"
        return Projection2d.apply(image, self._host(), self._prepare_angles(angles, image))

    def backprojection(self, sino: Tensor, angles: Tensor) -> Tensor:
        _, _, h, w = sino.shape
        v, = angles.shape
        assert (h, w) == (v, self.num_det), f"Expected input sino size {(v, self.num_det)}, but got {(h, w)}"
        return BackProjection2d.apply(sino, self._host(), self._prepare_angles(angles, sino))

    def backprojection_weighted(self, sino: Tensor, angles: Tensor) -> Tensor:
        _, _, h, w = sino.shape
        v, = angles.shape
        assert (h, w) == (v, self.num_det), f"Expected input sino size {(v, self.num_det)}, but got {(h, w)}"
        return WeightedBackProjection2d.apply(sino, self._host(), self._prepare_angles(angles, sino))

    def projection_t(self, sino: Tensor, angles: Tensor) -> Tensor:
        self._check_sino_angles(sino, angles)
        return ProjectionTranspose2d.apply(sino, self._host(), self._prepare_angles(angles, sino))

    def backprojection_t(self, image: Tensor, angles: Tensor) -> Tensor:
        _, _, h, w = image.shape
        assert (w, h) == self.image_size, f"Expected input image size {self.image_size[::-1]}, but got {(h, w)}"
        return BackProjectionTranspose2d.apply(image, self._host(), self._prepare_angles(angles, image))

    def backprojection_weighted_t(self, image: Tensor, angles: Tensor) -> Tensor:
        _, _, h, w = image.shape
        assert (w, h) == self.image_size, f"Expected input image size {self.image_size[::-1]}, but got {(h, w)}"
        return WeightedBackProjectionTranspose2d.apply(image, self._host(), self._prepare_angles(angles, image))

    projection_transpose = projection_t
    backprojection_transpose = backprojection_t
    weighted_backprojection_transpose = backprojection_weighted_t

    def system_matrix(self, angles: Tensor) -> Tensor:
        """Sparse COO projection matrix [V * Nv * Nu, D * H * W] (2D: [V * Nu,
        H * W]); the reference builds it on the CPU (system_matrix2d/3d,
        torch_binding.cpp:353-405).  Built here on the GPU; returned on the
        angles' device, so CPU angles give a CPU matrix as in the reference."""
        dev = angles.device if angles.is_cuda else torch.device("cuda", torch.cuda.current_device())
        m = _native.system_matrix(self._dim, self._host_geom.struct, angles, dev)
        return m if angles.is_cuda else m.cpu()

    get_sys_matrix = system_matrix

    def filtered_backprojection(self, sino: Tensor, angles: Tensor, filter: Optional[Tensor] = None,
                                filter_type: Optional[str] = None, redundant: Optional[bool] = None,
                                parker: bool = False) -> Tensor:
        return self._fbp(sino, angles, filter, filter_type, redundant, parker, rows_per_view=1)

    def apply_parker_weight(self, sino: Tensor, angles: Tensor) -> Tensor:
        return sino * self.parker_weight(angles).to(device=sino.device, dtype=sino.dtype)

    def parker_weight(self, angles: Tensor) -> Tensor:
        if self.scan_type not in ("flat", "arc") or angles.numel() < 2:
            return torch.ones((1, 1, angles.numel(), self.num_det), device=angles.device, dtype=angles.dtype)
        gamma = self._fan_angles(device=angles.device, dtype=angles.dtype)
        return parker_weights(angles, gamma, self.num_det).view(1, 1, angles.numel(), self.num_det)

    def _filter_generate(self, filter_type: str, dtype=None) -> Tensor:
        return filter_generate(self.num_det, self.det_size, filter_type, dtype)[None, None, None, :]

    def _make_cosine_weight(self, dtype=None) -> Tensor:
        dtype = dtype or torch.float32
        u = torch.arange(-self.num_det / 2 + 0.5, self.num_det / 2, 1.0, dtype=dtype)
        s = u * self.det_size + self.binshift
        if self.scan_type == "flat":
            w = self.iso_source / torch.sqrt(s * s + self.iso_source * self.iso_source)
        elif self.scan_type == "arc":
            w = torch.cos(s)
        else:
            w = torch.ones_like(s)
        return w.view(1, 1, 1, self.num_det)

    def _fan_angles(self, device=None, dtype=None) -> Tensor:
        dtype = dtype or torch.float32
        u = torch.arange(-self.num_det / 2 + 0.5, self.num_det / 2, 1.0, device=device, dtype=dtype)
        s = u * self.det_size + self.binshift
        if self.scan_type == "arc":
            return s
        if self.scan_type == "flat":
            return torch.atan2(s, torch.as_tensor(self.iso_source, device=device, dtype=dtype))
        return torch.zeros_like(s)

    def _check_sino_angles(self, sino: Tensor, angles: Tensor) -> None:
        if sino.ndim != 4:
            raise ValueError(f"Expected sino shape [B, C, V, Nu], got {tuple(sino.shape)}")
        if angles.ndim != 1:
            raise ValueError(f"Expected angles shape [V], got {tuple(angles.shape)}")
        if sino.shape[2] != angles.numel() or sino.shape[3] != self.num_det:
            raise ValueError(f"Expected sino shape [B, C, {angles.numel()}, {self.num_det}], got {tuple(sino.shape)}")


class Projector3d(_ProjectorBase):
    """Distance-driven 3D projector (parallel / cone-flat / cone-arc).

    Shapes: image [B, C, D, H, W], angles [V], sino [B, C, V, Nv, Nu].
    """
    _dim = 3

    def __init__(self, image_size, num_det=None, pix_size=None, det_size=None, iso_source: float = 0.0,
                 source_detector: float = 0.0, pixshift=0.0, binshift=0.0, scan_type: str = "flat",
                 filter_type: str = "ramp", trainable: bool = False, dtype=None) -> None:
        super().__init__()
        if isinstance(image_size, Volume3d):
            volume = image_size
            if isinstance(num_det, (ConeBeam3d, ParallelBeam3d)) and pix_size is None:
                pix_size = num_det
            if not isinstance(pix_size, (ConeBeam3d, ParallelBeam3d)):
                raise TypeError("When image_size is Volume3d, pix_size should be a Geometry3d object")
            geometry = pix_size
        else:
            if num_det is None or pix_size is None or det_size is None:
                raise TypeError("num_det, pix_size and det_size are required with the legacy constructor")
            volume = Volume3d(image_size, pix_size, pixshift)
            geometry = make_geometry3d(scan_type, num_det, det_size, iso_source, source_detector, binshift)
        scan = geometry.scan_type.lower().strip()
        if scan not in ("parallel", "flat", "arc"):
            raise ValueError(f"Unsupported 3D scan_type: {scan}")
        W, H, D = volume.size
        dx, dy, dz = volume.spacing
        shx, shy, shz = volume.shift
        self.volume = volume
        self.geometry = geometry
        self.image_size = (W, H, D)
        self.pix_size = (dx, dy, dz)
        self.num_det = tuple(geometry.detector.count)
        self.det_size = tuple(geometry.effective_det_spacing)
        self.binshift = tuple(geometry.effective_det_shift)
        self.pixshift = (shx * dx, shy * dy, shz * dz)
        self.scan_type = scan
        self.filter_type = filter_type.lower().strip()
        self.iso_source = float(getattr(geometry, "iso_source", 0.0))
        self.source_detector = float(getattr(geometry, "source_detector", 0.0))
        self._default_dtype = dtype or torch.float32
        packed = pack_options3d(volume, geometry)
        self._host_geom = HostGeometry(3, packed)
        self.register_buffer("options", torch.tensor(packed, dtype=self._default_dtype), persistent=False)
        w = self._make_cosine_weight(dtype=self._default_dtype)
        if trainable:
            self.weight = nn.Parameter(w.clone())
        else:
            self.register_buffer("weight", w, persistent=False)
        f = self._filter_generate(filter_type=self.filter_type, dtype=self._default_dtype)
        if trainable:
            self.filter = nn.Parameter(f.clone())
        else:
            self.register_buffer("filter", f, persistent=False)

    def _num_u(self) -> int:
        return self.num_det[0]

    def forward(self, image: Tensor, angles: Tensor) -> Tensor:
        return self.projection(image, angles)

    def projection(self, image: Tensor, angles: Tensor) -> Tensor:
        self._check_image(image)
        return Projection3d.apply(image, self._host(), self._prepare_angles(angles, image))

    def projection_t(self, sino: Tensor, angles: Tensor) -> Tensor:
        self._check_sino_angles(sino, angles)
        return ProjectionTranspose3d.apply(sino, self._host(), self._prepare_angles(angles, sino))

    def backprojection(self, sino: Tensor, angles: Tensor) -> Tensor:
        self._check_sino_angles(sino, angles)
        return BackProjection3d.apply(sino, self._host(), self._prepare_angles(angles, sino))

    def backprojection_weighted(self, sino: Tensor, angles: Tensor) -> Tensor:
        self._check_sino_angles(sino, angles)
        return WeightedBackProjection3d.apply(sino, self._host(), self._prepare_angles(angles, sino))

    def backprojection_t(self, image: Tensor, angles: Tensor) -> Tensor:
        self._check_image(image)
        return BackProjectionTranspose3d.apply(image, self._host(), self._prepare_angles(angles, image))

    def backprojection_weighted_t(self, image: Tensor, angles: Tensor) -> Tensor:
        self._check_image(image)
        return WeightedBackProjectionTranspose3d.apply(image, self._host(), self._prepare_angles(angles, image))

    def system_matrix(self, angles: Tensor) -> Tensor:
        """Sparse COO projection matrix [V * Nv * Nu, D * H * W] (2D: [V * Nu,
        H * W]); the reference builds it on the CPU (system_matrix2d/3d,
        torch_binding.cpp:353-405).  Built here on the GPU; returned on the
        angles' device, so CPU angles give a CPU matrix as in the reference."""
        dev = angles.device if angles.is_cuda else torch.device("cuda", torch.cuda.current_device())
        m = _native.system_matrix(self._dim, self._host_geom.struct, angles, dev)
        return m if angles.is_cuda else m.cpu()

    get_sys_matrix = system_matrix
    projection_transpose = projection_t
    backprojection_transpose = backprojection_t
    weighted_backprojection_transpose = backprojection_weighted_t

    def filtered_backprojection(self, sino: Tensor, angles: Tensor, filter: Optional[Tensor] = None,
                                filter_type: Optional[str] = None, redundant: Optional[bool] = None,
                                parker: bool = False) -> Tensor:
        """FDK: in-plane cosine weight (projector3d.py:233-246, no v term),
        u-filter, weighted backprojection, x mean angle step (/2 when
        redundant)."""
        return self._fbp(sino, angles, filter, filter_type, redundant, parker, rows_per_view=self.num_det[1])

    def parker_weight(self, angles: Tensor) -> Tensor:
        Nu = self.num_det[0]
        if angles.numel() < 2 or self.scan_type == "parallel":
            return torch.ones((1, 1, angles.numel(), 1, Nu), device=angles.device, dtype=angles.dtype)
        gamma = self._fan_angles(device=angles.device, dtype=angles.dtype)
        return parker_weights(angles, gamma, Nu).view(1, 1, angles.numel(), 1, Nu)

    def _filter_generate(self, filter_type: str, dtype=None) -> Tensor:
        return filter_generate(self.num_det[0], self.det_size[0], filter_type, dtype)[None, None, None, None, :]

    def _make_cosine_weight(self, dtype=None) -> Tensor:
        dtype = dtype or torch.float32
        Nu, du, shu = self.num_det[0], self.det_size[0], self.binshift[0]
        u = torch.arange(-Nu / 2 + 0.5, Nu / 2, 1.0, dtype=dtype)
        s = u * du + shu
        if self.scan_type == "parallel":
            return torch.ones((1, 1, 1, 1, Nu), dtype=dtype)
        if self.scan_type == "flat":
            w = self.iso_source / torch.sqrt(s * s + self.iso_source * self.iso_source)
        else:
            w = torch.cos(s)
        return w.view(1, 1, 1, 1, Nu)

    def _fan_angles(self, device=None, dtype=None) -> Tensor:
        dtype = dtype or torch.float32
        Nu, du, shu = self.num_det[0], self.det_size[0], self.binshift[0]
        u = torch.arange(-Nu / 2 + 0.5, Nu / 2, 1.0, device=device, dtype=dtype)
        s = u * du + shu
        if self.scan_type in ("parallel", "arc"):
            return s
        return torch.atan2(s, torch.as_tensor(self.iso_source, device=device, dtype=dtype))

    def _check_image(self, image: Tensor) -> None:
        if image.ndim != 5:
            raise ValueError(f"Expected image shape [B, C, D, H, W], got {tuple(image.shape)}")
        W, H, D = self.image_size
        if tuple(image.shape[2:]) != (D, H, W):
            raise ValueError(f"Expected image shape [B, C, {D}, {H}, {W}], got {tuple(image.shape)}")

    def _check_sino_angles(self, sino: Tensor, angles: Tensor) -> None:
        if sino.ndim != 5:
            raise ValueError(f"Expected sino shape [B, C, V, Nv, Nu], got {tuple(sino.shape)}")
        if angles.ndim != 1:
            raise ValueError(f"Expected angles shape [V], got {tuple(angles.shape)}")
        Nu, Nv = self.num_det
        if sino.shape[2] != angles.numel() or sino.shape[3] != Nv or sino.shape[4] != Nu:
            raise ValueError(f"Expected sino shape [B, C, {angles.numel()}, {Nv}, {Nu}], got {tuple(sino.shape)}")


class HelicalProjector3d(nn.Module):
    """Distance-driven helical cone-beam projector, arc detector
    (xrecon/projector/projector3d.py:289-576 of the reference).

    Shapes: image [B, C, D, H, W], angles [V], sino [B, C, V, Nv, Nu],
    source_pos [4, V] = (source_z, shift_radius, shift_angle, shift_z); when
    ``source_pos`` is omitted the source rises by ``pitch`` per turn from
    ``z0`` (:meth:`source_position`).  Operators run in float32, as in the
    reference.
    """

    _VIEW_MODES = {"auto": 0, "half": 1, "halfscan": 1, "half_scan": 1, "short": 1, "short_scan": 1,
                   "one": 2, "one_turn": 2, "1turn": 2, "full": 2, "full_scan": 2,
                   "fixed": 3, "turns": 3, "multi": 3, "multi_turn": 3}
    _WEIGHT_MODES = {"legacy": 0, "2d": 0, "redundancy": 0, "tang": 1, "tang3d": 1, "3d": 1, "cone": 1}

    def __init__(self, image_size, num_det=None, pix_size=None, det_size=None, iso_source: float = 0.0,
                 source_detector: float = 0.0, pixshift=0.0, binshift=0.0, scan_type: str = "arc",
                 pitch: float = 0.0, z0: float = 0.0, helical_view_mode: str = "one_turn",
                 helical_view_turns: float = 0.0, helical_halfscan_coef: float = 1.0,
                 helical_weight_mode: str = "2d", helical_tang_k: float = 5.0, helical_tang_blend: float = 0.0,
                 filter_type: str = "ramp", trainable: bool = False, dtype=None) -> None:
        super().__init__()
        if isinstance(image_size, Volume3d):
            volume = image_size
            if isinstance(num_det, HelicalConeBeam3d) and pix_size is None:
                pix_size = num_det
            if not isinstance(pix_size, HelicalConeBeam3d):
                raise TypeError("When image_size is Volume3d, pix_size should be a HelicalConeBeam3d object")
            geometry = pix_size
        else:
            if num_det is None or pix_size is None or det_size is None:
                raise TypeError("num_det, pix_size and det_size are required with the legacy constructor")
            volume = Volume3d(image_size, pix_size, pixshift)
            geometry = HelicalConeBeam3d(Detector3d(num_det, det_size, binshift), iso_source, source_detector,
                                         scan_type, pitch=pitch, z0=z0)
        scan = geometry.scan_type.lower().strip()
        if scan != "arc":
            raise NotImplementedError(
                "Direct helical projection/backprojection currently supports arc detector geometry only")
        W, H, D = volume.size
        dx, dy, dz = volume.spacing
        shx, shy, shz = volume.shift
        Nu, Nv = geometry.detector.count
        du, dv = geometry.effective_det_spacing
        shu, shv = geometry.effective_det_shift
        self.volume = volume
        self.geometry = geometry
        self.image_size = (W, H, D)
        self.pix_size = (dx, dy, dz)
        self.num_det = (Nu, Nv)
        self.det_size = (du, dv)
        self.binshift = (shu, shv)
        self.pixshift = (shx * dx, shy * dy, shz * dz)
        self.scan_type = scan
        self.filter_type = filter_type.lower().strip()
        self.iso_source = float(geometry.iso_source)
        self.source_detector = float(geometry.source_detector)
        self.pitch = float(geometry.pitch)
        self.z0 = float(geometry.z0)
        self.helical_view_mode = self._view_mode_id(helical_view_mode)
        self.helical_weight_mode = self._weight_mode_id(helical_weight_mode)
        self.helical_view_turns = float(helical_view_turns)
        self.helical_halfscan_coef = float(helical_halfscan_coef)
        self.helical_tang_k = float(helical_tang_k)
        self.helical_tang_blend = float(helical_tang_blend)
        self._default_dtype = dtype or torch.float32
        packed = [W, H, D, Nu, Nv, dx, dy, dz, du, dv, self.iso_source, self.source_detector,
                  self.pixshift[0], self.pixshift[1], self.pixshift[2], shu, shv, geometry.scan_id,
                  self.helical_view_mode, self.helical_weight_mode, self.helical_view_turns,
                  self.helical_halfscan_coef, self.helical_tang_k, self.helical_tang_blend]
        self._host_geom = HelicalHostGeometry(packed)
        self.register_buffer("options", torch.tensor(packed, dtype=self._default_dtype), persistent=False)
        w = self._make_weight(dtype=self._default_dtype)
        if trainable:
            self.weight = nn.Parameter(w.clone())
        else:
            self.register_buffer("weight", w, persistent=False)
        f = self._filter_generate(filter_type=self.filter_type, dtype=self._default_dtype)
        if trainable:
            self.filter = nn.Parameter(f.clone())
        else:
            self.register_buffer("filter", f, persistent=False)

    def forward(self, image: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None) -> Tensor:
        return self.projection(image, angles, source_pos)

    def source_position(self, angles: Tensor, ref: Optional[Tensor] = None) -> Tensor:
        """[4, V]: source z = z0 + pitch (beta - beta_0) / (2 pi), no shifts
        (projector3d.py:410-419)."""
        ref = angles if ref is None else ref
        angles = self._prepare_angles(angles, ref)
        if angles.numel() == 0:
            return angles.new_zeros((4, 0))
        source_z = self.z0 + self.pitch * (angles - angles[0]) / (2.0 * math.pi)
        shifts = angles.new_zeros((3, angles.numel()))
        return torch.cat((source_z.view(1, -1), shifts), dim=0).contiguous()

    def projection(self, image: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None) -> Tensor:
        self._check_image(image)
        angles = self._prepare_angles(angles, image)
        sp = self._prepare_source_pos(source_pos, angles, image)
        return ProjectionHelical3d.apply(image, self._host_geom, angles, sp)

    def projection_t(self, sino: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None) -> Tensor:
        self._check_sino_angles(sino, angles)
        angles = self._prepare_angles(angles, sino)
        sp = self._prepare_source_pos(source_pos, angles, sino)
        return ProjectionTransposeHelical3d.apply(sino, self._host_geom, angles, sp)

    def backprojection(self, sino: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None) -> Tensor:
        self._check_sino_angles(sino, angles)
        angles = self._prepare_angles(angles, sino)
        sp = self._prepare_source_pos(source_pos, angles, sino)
        return BackProjectionHelical3d.apply(sino, self._host_geom, angles, sp)

    def backprojection_weighted(self, sino: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None) -> Tensor:
        self._check_sino_angles(sino, angles)
        angles = self._prepare_angles(angles, sino)
        sp = self._prepare_source_pos(source_pos, angles, sino)
        return WeightedBackProjectionHelical3d.apply(sino, self._host_geom, angles, sp)

    def backprojection_t(self, image: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None) -> Tensor:
        self._check_image(image)
        angles = self._prepare_angles(angles, image)
        sp = self._prepare_source_pos(source_pos, angles, image)
        return BackProjectionTransposeHelical3d.apply(image, self._host_geom, angles, sp)

    def backprojection_weighted_t(self, image: Tensor, angles: Tensor,
                                  source_pos: Optional[Tensor] = None) -> Tensor:
        self._check_image(image)
        angles = self._prepare_angles(angles, image)
        sp = self._prepare_source_pos(source_pos, angles, image)
        return WeightedBackProjectionTransposeHelical3d.apply(image, self._host_geom, angles, sp)

    projection_transpose = projection_t
    backprojection_transpose = backprojection_t
    weighted_backprojection_transpose = backprojection_weighted_t
    backprojection_w = backprojection_weighted

    def filtered_backprojection(self, sino: Tensor, angles: Tensor, source_pos: Optional[Tensor] = None,
                                filter: Optional[Tensor] = None, filter_type: Optional[str] = None) -> Tensor:
        """Helical FDK (projector3d.py:465-481): cell weight [Nv, Nu], u-filter,
        weighted backprojection, x mean angle step (no redundancy halving)."""
        self._check_sino_angles(sino, angles)
        angles = self._prepare_angles(angles, sino)
        sp = self._prepare_source_pos(source_pos, angles, sino)
        if filter is not None:
            filt = filter
        elif filter_type is None or filter_type.lower() == self.filter_type:
            filt = self.filter
        else:
            filt = self._filter_generate(filter_type.lower(), dtype=sino.dtype).to(sino.device)
        Nu, Nv = self.num_det
        V = angles.numel()
        wt = self.weight
        needs_grad = torch.is_grad_enabled() and (
            sino.requires_grad or (isinstance(filt, Tensor) and filt.requires_grad) or wt.requires_grad)
        scale = mean_angle_step(angles)
        if needs_grad:
            sw = sino * wt.to(device=sino.device, dtype=sino.dtype)
            ones = torch.ones(Nu, device=sino.device, dtype=torch.float32)
            filtered = _FilterRows.apply(sw.to(torch.float32), ones, filt, None, V, Nv)
            recon = self.backprojection_weighted(filtered.contiguous(), angles, sp)
            return recon * scale.to(device=recon.device, dtype=recon.dtype)
        with torch.no_grad():
            s = sino if sino.is_contiguous() else sino.contiguous()
            # the [Nv, Nu] cell weight enters as the per-row weight of the
            # fused filter (one "view" per detector row)
            filtered = _native.fbp_filter(s, nview=Nv, rows_per_view=1, cosw=None,
                                          filt=filt.detach().reshape(-1),
                                          parker=wt.detach().reshape(Nv, Nu))
            recon = self.backprojection_weighted(filtered, angles, sp)
            return recon * scale.to(device=recon.device, dtype=recon.dtype)

    helical_fdk = filtered_backprojection

    @classmethod
    def _view_mode_id(cls, mode: str) -> int:
        key = str(mode).lower().strip()
        if key not in cls._VIEW_MODES:
            raise ValueError(f"Unsupported helical_view_mode: {mode}")
        return cls._VIEW_MODES[key]

    @classmethod
    def _weight_mode_id(cls, mode: str) -> int:
        key = str(mode).lower().strip()
        if key not in cls._WEIGHT_MODES:
            raise ValueError(f"Unsupported helical_weight_mode: {mode}")
        return cls._WEIGHT_MODES[key]

    def _filter_generate(self, filter_type: str, dtype=None) -> Tensor:
        return filter_generate(self.num_det[0], self.det_size[0], filter_type, dtype)[None, None, None, None, :]

    def _make_weight(self, dtype=None) -> Tensor:
        """SOD / |ray| of every cell (projector3d.py:535-545)."""
        dtype = dtype or torch.float32
        Nu, Nv = self.num_det
        du, dv = self.det_size
        shu, shv = self.binshift
        u = torch.arange(-Nu / 2 + 0.5, Nu / 2, 1.0, dtype=dtype) * du + shu
        v = torch.arange(-Nv / 2 + 0.5, Nv / 2, 1.0, dtype=dtype) * dv + shv
        col = torch.tan(u) * self.iso_source
        row = v * self.iso_source / self.source_detector
        w = self.iso_source / torch.sqrt(row[:, None].pow(2) + col[None, :].pow(2)
                                         + self.iso_source * self.iso_source)
        return w.view(1, 1, 1, Nv, Nu)

    def _check_image(self, image: Tensor) -> None:
        if image.ndim != 5:
            raise ValueError(f"Expected image shape [B, C, D, H, W], got {tuple(image.shape)}")
        W, H, D = self.image_size
        if tuple(image.shape[2:]) != (D, H, W):
            raise ValueError(f"Expected image shape [B, C, {D}, {H}, {W}], got {tuple(image.shape)}")

    def _check_sino_angles(self, sino: Tensor, angles: Tensor) -> None:
        if sino.ndim != 5:
            raise ValueError(f"Expected sino shape [B, C, V, Nv, Nu], got {tuple(sino.shape)}")
        if angles.ndim != 1:
            raise ValueError(f"Expected angles shape [V], got {tuple(angles.shape)}")
        Nu, Nv = self.num_det
        if sino.shape[2] != angles.numel() or sino.shape[3] != Nv or sino.shape[4] != Nu:
            raise ValueError(f"Expected sino shape [B, C, {angles.numel()}, {Nv}, {Nu}], got {tuple(sino.shape)}")

    def _prepare_source_pos(self, source_pos: Optional[Tensor], angles: Tensor, ref: Tensor) -> Tensor:
        if source_pos is None:
            return self.source_position(angles, ref)
        source_pos = source_pos.to(device=ref.device, dtype=ref.dtype).contiguous()
        if source_pos.shape != (4, angles.numel()):
            raise ValueError(f"Expected source_pos shape [4, {angles.numel()}], got {tuple(source_pos.shape)}")
        return source_pos

    @staticmethod
    def _prepare_angles(angles: Tensor, ref: Tensor) -> Tensor:
        return angles.to(device=ref.device, dtype=ref.dtype).contiguous()

    @staticmethod
    def _mean_angle_step(angles: Tensor) -> Tensor:
        return mean_angle_step(angles)


projector2d = Projector2d
projector3d = Projector3d
