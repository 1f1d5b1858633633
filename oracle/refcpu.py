"""The reference's own CPU operators (XRecon ``src/cpu``), loaded from
``oracle/_ref/libxrecon_ref_cpu.so`` built by ``build_oracle.build_ref``.

TEST INFRASTRUCTURE ONLY (test comparisons and the CPU reference arm of ``bench.py``).

:class:`RefXreconC` mirrors the surface of the reference's ``xrecon_C``
extension (``src/api/torch_binding.cpp:615-638``) on CPU tensors, so the
reference's own Python package can run on top of its own C++ CPU kernels when
the reference tree is importable (fixture generation in this container).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import build_oracle
from .oracle import OPS, SINO_OUT, unpack2d, unpack3d

_lib = None


def available() -> bool:
    try:
        _load()
        return True
    except (OSError, RuntimeError):
        return False


def _load():
    global _lib
    if _lib is None:
        so = build_oracle.build_ref()
        if so is None or not so.exists():
            raise RuntimeError("reference CPU library not built (oracle/_ref)")
        lib = ctypes.CDLL(str(so))
        lib.xr_ref_dd2d.restype = ctypes.c_int
        lib.xr_ref_dd2d.argtypes = ([ctypes.c_int] + [ctypes.POINTER(ctypes.c_float)] * 3 +
                                    [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 4 +
                                    [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 4 +
                                    [ctypes.c_int, ctypes.c_int])
        lib.xr_ref_dd3d.restype = ctypes.c_int
        lib.xr_ref_dd3d.argtypes = ([ctypes.c_int] + [ctypes.POINTER(ctypes.c_float)] * 3 +
                                    [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                     ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int, ctypes.c_int])
        lib.xr_ref_sysmat2d.restype = ctypes.c_longlong
        lib.xr_ref_sysmat2d.argtypes = ([ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int] +
                                        [ctypes.c_float] * 4 + [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 4 +
                                        [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_longlong])
        lib.xr_ref_sysmat3d.restype = ctypes.c_longlong
        lib.xr_ref_sysmat3d.argtypes = ([ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                         ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_longlong])
        _lib = lib
    return _lib


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def dd2d(op: str, x, options, angles) -> np.ndarray:
    g = unpack2d(options)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    V = ang.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float32)
    B, C = x.shape[:2]
    img_shape = (B, C, g["H"], g["W"])
    sino_shape = (B, C, V, g["Nu"])
    if op in SINO_OUT:
        image, proj = x, np.zeros(sino_shape, np.float32)
    else:
        image, proj = np.zeros(img_shape, np.float32), x
    rc = _load().xr_ref_dd2d(OPS[op], _fp(image), _fp(proj), _fp(ang), g["W"], g["H"],
                             g["dx"], g["dy"], g["shx"], g["shy"], g["type"], g["Nu"],
                             g["du"], g["shu"], g["SOD"], g["SDD"], B * C, V)
    if rc != 0:
        raise RuntimeError(f"reference dd2d failed ({rc})")
    return proj if op in SINO_OUT else image


def dd3d(op: str, x, options, angles) -> np.ndarray:
    g = unpack3d(options)
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    V = ang.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float32)
    B, C = x.shape[:2]
    img_shape = (B, C, g["D"], g["H"], g["W"])
    sino_shape = (B, C, V, g["Nv"], g["Nu"])
    if op in SINO_OUT:
        image, proj = x, np.zeros(sino_shape, np.float32)
    else:
        image, proj = np.zeros(img_shape, np.float32), x
    ni = np.array([g["W"], g["H"], g["D"], g["Nu"], g["Nv"]], dtype=np.int32)
    fv = np.array([g["dx"], g["dy"], g["dz"], g["shx"], g["shy"], g["shz"]], dtype=np.float32)
    fg = np.array([g["du"], g["dv"], g["shu"], g["shv"], g["SOD"], g["SDD"]], dtype=np.float32)
    rc = _load().xr_ref_dd3d(OPS[op], _fp(image), _fp(proj), _fp(ang),
                             ni.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _fp(fv), _fp(fg),
                             g["type"], B * C, V)
    if rc != 0:
        raise RuntimeError(f"reference dd3d failed ({rc})")
    return proj if op in SINO_OUT else image


class RefXreconC:
    """``xrecon_C``-shaped facade over the reference CPU kernels (CPU tensors
    only), binding names as in torch_binding.cpp:615-638."""

    def __init__(self):
        import torch
        self._torch = torch

    def _wrap(self, fn, op, x, options, angles):
        t = self._torch
        out = fn(op, x.detach().cpu().numpy(), options.detach().cpu().numpy(), angles.detach().cpu().numpy())
        return t.from_numpy(np.ascontiguousarray(out))

    def forward_projection2d(self, x, o, a): return self._wrap(dd2d, "A", x, o, a)
    def projection_transpose2d(self, x, o, a): return self._wrap(dd2d, "AT", x, o, a)
    def backward_projection2d(self, x, o, a): return self._wrap(dd2d, "B", x, o, a)
    def weighted_backward_projection2d(self, x, o, a): return self._wrap(dd2d, "BW", x, o, a)
    def backward_projection_transpose2d(self, x, o, a): return self._wrap(dd2d, "BT", x, o, a)
    def weighted_backward_projection_transpose2d(self, x, o, a): return self._wrap(dd2d, "BWT", x, o, a)
    back_projection2d = backward_projection2d
    weighted_back_projection2d = weighted_backward_projection2d

    def forward_projection3d(self, x, o, a): return self._wrap(dd3d, "A", x, o, a)
    def projection_transpose3d(self, x, o, a): return self._wrap(dd3d, "AT", x, o, a)
    def backward_projection3d(self, x, o, a): return self._wrap(dd3d, "B", x, o, a)
    def weighted_backward_projection3d(self, x, o, a): return self._wrap(dd3d, "BW", x, o, a)
    def backward_projection_transpose3d(self, x, o, a): return self._wrap(dd3d, "BT", x, o, a)
    def weighted_backward_projection_transpose3d(self, x, o, a): return self._wrap(dd3d, "BWT", x, o, a)


def system_matrix(dim: int, options, angles):
    """The reference's system_matrix2d_cpu / system_matrix3d_cpu triplets
    (rows, cols, vals) as numpy arrays, unsorted, and the matrix shape."""
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    V = ang.shape[0]
    L = _load()
    cap = 0
    while True:
        rows = np.zeros(max(cap, 1), np.int64)
        cols = np.zeros(max(cap, 1), np.int64)
        vals = np.zeros(max(cap, 1), np.float32)
        args = (rows.ctypes.data, cols.ctypes.data, vals.ctypes.data, cap)
        if dim == 2:
            g = unpack2d(options)
            n = L.xr_ref_sysmat2d(_fp(ang), g["W"], g["H"], g["dx"], g["dy"], g["shx"], g["shy"], g["type"],
                                  g["Nu"], g["du"], g["shu"], g["SOD"], g["SDD"], V, *args)
            shape = (V * g["Nu"], g["H"] * g["W"])
        else:
            g = unpack3d(options)
            ni = np.array([g["W"], g["H"], g["D"], g["Nu"], g["Nv"]], dtype=np.int32)
            fv = np.array([g["dx"], g["dy"], g["dz"], g["shx"], g["shy"], g["shz"]], dtype=np.float32)
            fg = np.array([g["du"], g["dv"], g["shu"], g["shv"], g["SOD"], g["SDD"]], dtype=np.float32)
            n = L.xr_ref_sysmat3d(_fp(ang), ni.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _fp(fv), _fp(fg),
                                  g["type"], V, *args)
            shape = (V * g["Nv"] * g["Nu"], g["D"] * g["H"] * g["W"])
        if n < 0:
            raise RuntimeError("reference system matrix failed")
        if n <= cap:
            return rows[:n], cols[:n], vals[:n], shape
        cap = int(n)
