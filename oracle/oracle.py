"""FP64 CPU oracle for the distance-driven projector path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product package never
does.

* :func:`dd2d` / :func:`dd3d` / :func:`helical3d` run the C restatement
  ``dd_oracle.c`` in double precision.  They take the reference's packed ``options`` vector (12 entries
  in 2D, 18 in 3D) and unpack it exactly as the reference binding does
  (XRecon ``src/api/torch_binding.cpp:62-124``), so both sides see identical
  float32 parameter values.
* :func:`filtered_backprojection2d` / :func:`filtered_backprojection3d`
  restate the reference's FBP / FDK pipelines (``xrecon/projector/
  projector.py:176-313`` and ``projector3d.py:165-287``) in numpy float64,
  with the filter correlation evaluated directly.
"""
from __future__ import annotations

import contextlib
import ctypes
import math
from pathlib import Path

import numpy as np

from . import build_oracle

OPS = {"A": 0, "AT": 1, "B": 2, "BT": 3, "BW": 4, "BWT": 5}
SINO_OUT = {"A", "BT", "BWT"}

_lib = None


def _load():
    global _lib
    if _lib is None:
        so = build_oracle.ORACLE_SO
        if not so.exists():
            build_oracle.build_oracle()
        lib = ctypes.CDLL(str(so))
        for name in ("xo_dd2d", "xo_dd3d"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int]
        lib.xo_set_arc_exact.restype = None
        lib.xo_set_arc_exact.argtypes = [ctypes.c_int]
        lib.xo_set_tan_rounding.restype = None
        lib.xo_set_tan_rounding.argtypes = [ctypes.c_int]
        dp = ctypes.POINTER(ctypes.c_double)
        lib.xo_helical3d.restype = ctypes.c_int
        lib.xo_helical3d.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), dp, dp, dp, dp, dp,
                                     ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                     ctypes.c_int, ctypes.c_int]
        _lib = lib
    return _lib


@contextlib.contextmanager
def tan_rounding(correctly_rounded: bool):
    """Within the block, the arc operators take the CUDA path's arithmetic:
    the axis mapping uses tan rounded correctly to float32 instead of the C
    library's tanf (the reference CPU path's, the default; glibc's is off by
    one unit for about 4 % of arguments), and B / Bw take their chained
    column boundaries linearised around the direct ones."""
    lib = _load()
    lib.xo_set_tan_rounding(int(correctly_rounded))
    try:
        yield
    finally:
        lib.xo_set_tan_rounding(0)


def _p(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def unpack2d(options):
    """Same field order as torch_binding.cpp:62-79."""
    o = np.asarray(options, dtype=np.float32)
    return dict(W=int(o[0]), H=int(o[1]), Nu=int(o[2]), dx=o[3], dy=o[4], du=o[5],
                SOD=o[6], SDD=o[7], shx=o[8], shy=o[9], shu=o[10], type=int(o[11]))


def unpack3d(options):
    """Same field order as torch_binding.cpp:82-124 (helical fields ignored)."""
    o = np.asarray(options, dtype=np.float32)
    return dict(W=int(o[0]), H=int(o[1]), D=int(o[2]), Nu=int(o[3]), Nv=int(o[4]),
                dx=o[5], dy=o[6], dz=o[7], du=o[8], dv=o[9], SOD=o[10], SDD=o[11],
                shx=o[12], shy=o[13], shz=o[14], shu=o[15], shv=o[16], type=int(o[17]))


def dd2d(op: str, x, options, angles, arc_exact: bool = False):
    """Apply a 2D operator.  x: [B, C, H, W] (image in) or [B, C, V, Nu]
    (sinogram in); returns float64 ndarray of the output shape.  Arc
    boundary angles are rounded to float32 as the reference forms them
    (``dd_oracle.c::arc_angle``) unless ``arc_exact``."""
    g = unpack2d(options)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    V = ang.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float64)
    B, C = x.shape[:2]
    out_shape = (B, C, V, g["Nu"]) if op in SINO_OUT else (B, C, g["H"], g["W"])
    out = np.zeros(out_shape, dtype=np.float64)
    ni = np.array([g["W"], g["H"], g["Nu"]], dtype=np.int32)
    fv = np.array([g["dx"], g["dy"], g["shx"], g["shy"]], dtype=np.float64)
    fg = np.array([g["du"], g["shu"], g["SOD"], g["SDD"]], dtype=np.float64)
    _load().xo_set_arc_exact(int(arc_exact))
    rc = _load().xo_dd2d(OPS[op], _p(ni, ctypes.c_int), _p(fv, ctypes.c_double), _p(fg, ctypes.c_double),
                         g["type"], _p(x, ctypes.c_double), _p(out, ctypes.c_double),
                         _p(ang, ctypes.c_float), B * C, V)
    if rc != 0:
        raise RuntimeError(f"oracle dd2d failed with status {rc}")
    return out


def dd3d(op: str, x, options, angles, arc_exact: bool = False):
    """Apply a 3D operator.  x: [B, C, D, H, W] or [B, C, V, Nv, Nu].  Arc
    boundary angles as in :func:`dd2d`."""
    g = unpack3d(options)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    V = ang.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float64)
    B, C = x.shape[:2]
    out_shape = (B, C, V, g["Nv"], g["Nu"]) if op in SINO_OUT else (B, C, g["D"], g["H"], g["W"])
    out = np.zeros(out_shape, dtype=np.float64)
    ni = np.array([g["W"], g["H"], g["D"], g["Nu"], g["Nv"]], dtype=np.int32)
    fv = np.array([g["dx"], g["dy"], g["dz"], g["shx"], g["shy"], g["shz"]], dtype=np.float64)
    fg = np.array([g["du"], g["dv"], g["shu"], g["shv"], g["SOD"], g["SDD"]], dtype=np.float64)
    _load().xo_set_arc_exact(int(arc_exact))
    rc = _load().xo_dd3d(OPS[op], _p(ni, ctypes.c_int), _p(fv, ctypes.c_double), _p(fg, ctypes.c_double),
                         g["type"], _p(x, ctypes.c_double), _p(out, ctypes.c_double),
                         _p(ang, ctypes.c_float), B * C, V)
    if rc != 0:
        raise RuntimeError(f"oracle dd3d failed with status {rc}")
    return out


def unpack_helical(options):
    """Helical fields of the 3D options vector with the binding's defaults
    (torch_binding.cpp:103-108): view_mode, weight_mode, view_turns,
    halfscan_coef, tang_k, tang_blend."""
    o = np.asarray(options, dtype=np.float32)
    dflt = [2.0, 0.0, 0.0, 1.0, 5.0, 0.0]
    vals = [float(o[18 + i]) if o.size > 18 + i else dflt[i] for i in range(6)]
    vals[0], vals[1] = float(int(vals[0])), float(int(vals[1]))
    return vals


def helical3d(op: str, x, options, angles, source_pos, window_quotient_up: bool = False):
    """Apply a helical arc-detector operator (the reference's
    src/kernels/helical_arc3d.cu).  x: [B, C, D, H, W] or [B, C, V, Nv, Nu];
    source_pos: [4, V] (source_z, shift_radius, shift_angle, shift_z).

    ``window_quotient_up`` takes the view-window length ceil(span / |dbeta|)
    of a quotient moved one float ulp up: the reference, built with
    --use_fast_math, evaluates that division approximately, and at an exact
    integer quotient (whole views per turn) its window came out one view
    longer than the exact formula gives.  Only the pin against the
    reference's recorded outputs uses it."""
    g = unpack3d(options)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    V = ang.shape[0]
    sp = np.ascontiguousarray(source_pos, dtype=np.float32)
    if sp.shape != (4, V):
        raise ValueError(f"source_pos must be [4, {V}], got {sp.shape}")
    x = np.ascontiguousarray(x, dtype=np.float64)
    B, C = x.shape[:2]
    out_shape = (B, C, V, g["Nv"], g["Nu"]) if op in SINO_OUT else (B, C, g["D"], g["H"], g["W"])
    out = np.zeros(out_shape, dtype=np.float64)
    ni = np.array([g["W"], g["H"], g["D"], g["Nu"], g["Nv"]], dtype=np.int32)
    fv = np.array([g["dx"], g["dy"], g["dz"], g["shx"], g["shy"], g["shz"]], dtype=np.float64)
    fg = np.array([g["du"], g["dv"], g["shu"], g["shv"], g["SOD"], g["SDD"]], dtype=np.float64)
    fo = np.array(unpack_helical(options) + [1.0 if window_quotient_up else 0.0], dtype=np.float64)
    rc = _load().xo_helical3d(OPS[op], _p(ni, ctypes.c_int), _p(fv, ctypes.c_double), _p(fg, ctypes.c_double),
                              _p(fo, ctypes.c_double), _p(x, ctypes.c_double), _p(out, ctypes.c_double),
                              _p(ang, ctypes.c_float), _p(sp, ctypes.c_float), B * C, V)
    if rc != 0:
        raise RuntimeError(f"oracle helical3d failed with status {rc}")
    return out


# ---------------------------------------------------------------- FBP / FDK

def ramp_filter(num_det: int, det_size: float) -> np.ndarray:
    """Spatial Ram-Lak kernel of length 2*Nu-1 (filters.py:19-32)."""
    x = np.arange(2 * num_det - 1) - num_det + 1
    f = np.zeros(2 * num_det - 1, dtype=np.float64)
    odd = (x % 2) != 0
    f[odd] = -1.0 / (math.pi ** 2 * det_size ** 2 * (x[odd].astype(np.float64) ** 2 + 1e-12))
    f[num_det - 1] = 1.0 / (4.0 * det_size ** 2)
    return f


def correlate_rows(sino: np.ndarray, filt: np.ndarray) -> np.ndarray:
    """out[..., i] = sum_j sino[..., j] * filt[j - i + Nu - 1]: the reference's
    conv2d/conv3d with padding Nu-1 along u (projector.py:201,
    projector3d.py:190; torch conv is cross-correlation)."""
    nu = sino.shape[-1]
    f = np.asarray(filt, dtype=np.float64).reshape(-1)
    assert f.shape[0] == 2 * nu - 1
    # T[j, i] = f[j - i + nu - 1]
    j = np.arange(nu)[:, None]
    i = np.arange(nu)[None, :]
    T = f[j - i + nu - 1]
    return np.asarray(sino, dtype=np.float64) @ T


def mean_angle_step(angles) -> float:
    """projector.py:303-313."""
    a = np.asarray(angles, dtype=np.float64)
    if a.size < 2:
        return 0.0
    d = np.diff(a)
    wrap = np.mod(d + math.pi, 2 * math.pi) - math.pi
    return float(np.abs(wrap).mean())


def cosine_weight(scan: str, nu: int, du_eff: float, shu_eff: float, sod: float) -> np.ndarray:
    """projector.py:255-277 / projector3d.py:233-246 (3D: in-plane only)."""
    u = np.arange(-nu / 2 + 0.5, nu / 2, 1.0, dtype=np.float64)
    s = u * du_eff + shu_eff
    if scan == "flat":
        return sod / np.sqrt(s * s + sod * sod)
    if scan == "arc":
        return np.cos(s)
    return np.ones_like(s)


def filtered_backprojection2d(sino, options, angles, weight, filt, redundant=True, parker=None):
    """Restates Projector2d.filtered_backprojection (projector.py:176-206)."""
    s = np.asarray(sino, dtype=np.float64)
    if parker is not None:
        s = s * np.asarray(parker, dtype=np.float64)
    s = s * np.asarray(weight, dtype=np.float64).reshape(-1)
    f = correlate_rows(s, filt)
    recon = dd2d("BW", f, options, angles) * mean_angle_step(angles)
    return recon / 2 if redundant else recon


def filtered_backprojection3d(sino, options, angles, weight, filt, redundant=True, parker=None):
    """Restates Projector3d.filtered_backprojection (projector3d.py:165-195)."""
    s = np.asarray(sino, dtype=np.float64)
    if parker is not None:
        s = s * np.asarray(parker, dtype=np.float64)
    s = s * np.asarray(weight, dtype=np.float64).reshape(-1)
    f = correlate_rows(s, filt)
    recon = dd3d("BW", f, options, angles) * mean_angle_step(angles)
    return recon / 2 if redundant else recon


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


# ---------------------------------------------------------------- rebinning

def rebin_grid(angles, Nu, iso_source, det_spacing, det_shift, detector_type, output_angles, Nt,
               output_det_spacing, output_det_shift):
    """Sampling grid of fan_to_parallel_rebin (xrecon/utils/rebin.py:67-95),
    in the reference's float32 arithmetic: [Vout, Nt, 2] (x: column, y: view)
    normalized for align_corners=True, and the bin centres t [Nt]."""
    f32 = np.float32
    a = np.asarray(angles, f32)
    oa = np.asarray(output_angles, f32)
    u = (np.arange(-Nu / 2 + 0.5, Nu / 2, 1.0).astype(f32) * f32(det_spacing) + f32(det_shift)).astype(f32)
    if detector_type == "arc":
        gext = np.abs(u).max()
    else:
        gext = np.arctan2(np.abs(u).max(), f32(iso_source)).astype(f32)
    max_t = f32(iso_source) * np.sin(gext).astype(f32)
    if output_det_spacing is None:
        output_det_spacing = float(f32(2.0) * max_t / f32(Nt)) if Nt > 0 else 1.0
    t = (np.arange(-Nt / 2 + 0.5, Nt / 2, 1.0).astype(f32) * f32(output_det_spacing) + f32(output_det_shift)).astype(f32)
    ratio = np.clip(t / f32(iso_source), f32(-1.0 + 1e-6), f32(1.0 - 1e-6)).astype(f32)
    gamma = np.arcsin(ratio).astype(f32)
    beta = (oa[:, None] - gamma[None, :]).astype(f32)
    uq = gamma if detector_type == "arc" else (np.tan(gamma).astype(f32) * f32(iso_source)).astype(f32)
    V = a.size
    step = f32(1.0) if V < 2 else np.diff(a).mean(dtype=f32)
    bidx = ((beta - a[0]) / step).astype(f32)
    ucoord = ((uq - f32(det_shift)) / f32(det_spacing) + f32(Nu / 2 - 0.5)).astype(f32)
    gy = (f32(2.0) * bidx / f32(max(V - 1, 1)) - f32(1.0)).astype(f32)
    gx = (f32(2.0) * ucoord[None, :] / f32(max(Nu - 1, 1)) - f32(1.0)).astype(f32)
    return np.stack([np.broadcast_to(gx, gy.shape), gy], axis=-1), t


def grid_sample_rows(sino5, grid):
    """Bilinear sampling of every [V, Nu] plane of sino5 [B, C, V, Nv, Nu] at
    grid [Vout, Nt, 2] (align_corners=True, zero padding), FP64:
    [B, C, Vout, Nv, Nt]."""
    s = np.asarray(sino5, np.float64)
    B, C, V, Nv, Nu = s.shape
    g = np.asarray(grid, np.float64)
    ix = (g[..., 0] + 1.0) / 2.0 * (Nu - 1)
    iy = (g[..., 1] + 1.0) / 2.0 * (V - 1)
    x0, y0 = np.floor(ix).astype(np.int64), np.floor(iy).astype(np.int64)
    out = np.zeros((B, C, g.shape[0], Nv, g.shape[1]))
    for dy, wy in ((0, y0 + 1 - iy), (1, iy - y0)):
        for dx, wx in ((0, x0 + 1 - ix), (1, ix - x0)):
            yy, xx = y0 + dy, x0 + dx
            ok = (yy >= 0) & (yy < V) & (xx >= 0) & (xx < Nu)
            val = s[:, :, np.clip(yy, 0, V - 1), :, np.clip(xx, 0, Nu - 1)]  # [Vout, Nt, B, C, Nv]
            val = np.moveaxis(val, (0, 1), (3, 4))                              # [B, C, Nv, Vout, Nt]
            out += np.moveaxis(val * (wx * wy * ok), 2, 3)
    return out


def fan_to_parallel_rebin(sino, angles, iso_source, det_spacing, det_shift=0.0, detector_type="arc",
                          output_angles=None, output_det_count=None, output_det_spacing=None,
                          output_det_shift=0.0):
    """FP64 restatement of the reference's fan_to_parallel_rebin
    (rebin.py:10-95): (parallel sinogram, output angles, t)."""
    s = np.asarray(sino)
    s5 = s[:, :, :, None, :] if s.ndim == 4 else s
    Nu = s5.shape[-1]
    oa = np.asarray(angles if output_angles is None else output_angles, np.float32)
    Nt = Nu if output_det_count is None else int(output_det_count)
    grid, t = rebin_grid(angles, Nu, iso_source, det_spacing, det_shift, detector_type, oa, Nt,
                         output_det_spacing, output_det_shift)
    out = grid_sample_rows(s5, grid)
    return (out[:, :, :, 0, :] if s.ndim == 4 else out), oa, t
