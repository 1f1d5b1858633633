"""Fan/cone -> parallel rebinning on the GPU.

Same functions, arguments and results as the reference's
``xrecon/utils/rebin.py`` (fan_to_parallel_rebin, helical_fan_to_parallel_rebin
and its alias helical_cone_to_parallel_rebin).  The sampling grid is built
with the reference's float32 steps (parallel bins t = SOD sin(gamma), views
beta = theta - gamma, normalized for align_corners=True), and the bilinear
sampling with zero padding that the reference delegates to
torch.nn.functional.grid_sample runs in this library's kernel
(``xr_rebin_parallel``).  With ``filt`` (2 Nt - 1 taps), the rebinned rows
are also filtered in the same pass, ready for a parallel-beam FBP.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import torch
from torch import Tensor

from . import _native


def _lib():
    L = _native.lib()
    if not getattr(L, "_rebin_ready", False):
        L.xr_rebin_parallel.restype = ctypes.c_int
        L.xr_rebin_parallel.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p] + [ctypes.c_int] * 4 + \
                                       [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L._rebin_ready = True
    return L


def rebin_grid(angles: Tensor, Nu: int, iso_source: float, det_spacing: float, det_shift: float,
               detector_type: str, output_angles: Tensor, Nt: int, output_det_spacing: Optional[float],
               output_det_shift: float) -> Tuple[Tensor, Tensor]:
    """The normalized sampling grid [Vout, Nt, 2] (x: detector column, y:
    view) and the parallel bin centres t [Nt], in the reference's float32
    arithmetic (rebin.py:67-95)."""
    dev, dt = angles.device, angles.dtype
    u = torch.arange(-Nu / 2 + 0.5, Nu / 2, device=dev, dtype=dt) * float(det_spacing) + float(det_shift)
    if detector_type == "arc":
        gamma_extent = u.abs().max()
    else:
        gamma_extent = torch.atan2(u.abs().max(), u.new_tensor(float(iso_source)))
    max_t = float(iso_source) * torch.sin(gamma_extent)
    if output_det_spacing is None:
        output_det_spacing = (2.0 * max_t / Nt).item() if Nt > 0 else 1.0
    t = torch.arange(-Nt / 2 + 0.5, Nt / 2, device=dev, dtype=dt) * float(output_det_spacing) + float(output_det_shift)
    gamma = torch.asin(torch.clamp(t / float(iso_source), min=-1.0 + 1e-6, max=1.0 - 1e-6))
    beta = output_angles[:, None] - gamma[None, :]
    u_query = gamma if detector_type == "arc" else torch.tan(gamma) * float(iso_source)
    V = angles.numel()
    step = angles.new_tensor(1.0) if V < 2 else torch.diff(angles).mean()
    beta_index = (beta - angles[0]) / step
    u_coord = (u_query - float(det_shift)) / float(det_spacing) + Nu / 2 - 0.5
    gy = 2.0 * beta_index / max(V - 1, 1) - 1.0
    gx = 2.0 * u_coord[None, :] / max(Nu - 1, 1) - 1.0
    return torch.stack((gx.expand_as(gy), gy), dim=-1).contiguous(), t


def fan_to_parallel_rebin(sino: Tensor, angles: Tensor, iso_source: float, det_spacing: float,
                          det_shift: float = 0.0, detector_type: str = "arc",
                          output_angles: Optional[Tensor] = None, output_det_count: Optional[int] = None,
                          output_det_spacing: Optional[float] = None, output_det_shift: float = 0.0,
                          filt: Optional[Tensor] = None) -> Tuple[Tensor, Tensor, Tensor]:
    """Rebin [B, C, V, Nu] or [B, C, V, Nv, Nu] fan/cone data to a parallel
    geometry along the detector columns; returns (parallel_sino,
    output_angles, output_t) as the reference.  ``filt`` (optional, [2 Nt -
    1]) also filters the rebinned rows in the same pass."""
    if sino.ndim not in (4, 5):
        raise ValueError(f"Expected sino shape [B,C,V,Nu] or [B,C,V,Nv,Nu], got {tuple(sino.shape)}")
    if angles.ndim != 1:
        raise ValueError(f"Expected angles shape [V], got {tuple(angles.shape)}")
    detector_type = detector_type.lower().strip()
    if detector_type not in {"arc", "flat"}:
        raise ValueError("detector_type should be 'arc' or 'flat'")
    _native._check_cuda("sino", sino)
    sino5 = sino[:, :, :, None, :] if sino.ndim == 4 else sino
    B, C, V, Nv, Nu = sino5.shape
    if V != angles.numel():
        raise ValueError(f"Expected {V} angles, got {angles.numel()}")
    dt = sino.dtype if sino.dtype == torch.float32 else torch.float32
    out_ang = (angles if output_angles is None else output_angles).to(device=sino.device, dtype=dt).contiguous()
    angles = angles.to(device=sino.device, dtype=dt).contiguous()
    Nt = Nu if output_det_count is None else int(output_det_count)
    grid, t = rebin_grid(angles, Nu, iso_source, det_spacing, det_shift, detector_type, out_ang, Nt,
                         output_det_spacing, output_det_shift)
    src = sino5.contiguous()
    if src.dtype not in _native.DTYPES:
        src = src.float()
    out = torch.empty((B, C, out_ang.numel(), Nv, Nt), dtype=torch.float32, device=sino.device)
    f = None
    if filt is not None:
        f = filt.to(device=sino.device, dtype=torch.float32).contiguous().reshape(-1)
        if f.numel() != 2 * Nt - 1:
            raise ValueError(f"filter must have 2*Nt-1 = {2 * Nt - 1} taps, got {f.numel()}")
    if out.numel():
        with torch.cuda.device(sino.device):
            rc = _lib().xr_rebin_parallel(src.data_ptr(), _native.DTYPES[src.dtype], out.data_ptr(), B * C, V, Nv, Nu,
                                          grid.data_ptr(), out_ang.numel(), Nt, None if f is None else f.data_ptr(),
                                          torch.cuda.current_stream(sino.device).cuda_stream)
        if rc != 0:
            _native._raise(rc, "xr_rebin_parallel")
    if sino.ndim == 4:
        out = out[:, :, :, 0, :]
    return out, out_ang, t


def helical_fan_to_parallel_rebin(sino: Tensor, angles: Tensor, source_z: Tensor, iso_source: float,
                                  det_spacing: float, det_shift: float = 0.0, detector_type: str = "arc",
                                  output_angles: Optional[Tensor] = None, output_det_count: Optional[int] = None,
                                  output_det_spacing: Optional[float] = None, output_det_shift: float = 0.0,
                                  filt: Optional[Tensor] = None) -> Tuple[Tensor, Tensor, Tensor, Tensor]:
    """Helical variant: also interpolates the source z position linearly onto
    the output angles (zero outside the input range), as the reference's
    helical_fan_to_parallel_rebin (rebin.py:97-168)."""
    if source_z.ndim != 1:
        raise ValueError(f"Expected source_z shape [V], got {tuple(source_z.shape)}")
    if source_z.numel() != angles.numel():
        raise ValueError(f"Expected source_z length {angles.numel()}, got {source_z.numel()}")
    out, out_ang, t = fan_to_parallel_rebin(sino, angles, iso_source, det_spacing, det_shift, detector_type,
                                            output_angles, output_det_count, output_det_spacing, output_det_shift,
                                            filt=filt)
    z = source_z.to(device=out.device, dtype=out.dtype).contiguous()
    a_in = angles.to(device=out.device, dtype=out.dtype).contiguous()
    if a_in.numel() < 2:
        return out, out_ang, t, z.expand_as(out_ang).contiguous()
    idx = (out_ang - a_in[0]) / torch.diff(a_in).mean()
    i0 = torch.floor(idx).to(torch.long)
    i1 = i0 + 1
    w = (idx - i0.to(idx.dtype)).clamp(0.0, 1.0)
    valid = (i0 >= 0) & (i1 < z.numel())
    zi = (1.0 - w) * z[i0.clamp(0, z.numel() - 1)] + w * z[i1.clamp(0, z.numel() - 1)]
    return out, out_ang, t, torch.where(valid, zi, torch.zeros_like(zi)).contiguous()


helical_cone_to_parallel_rebin = helical_fan_to_parallel_rebin
