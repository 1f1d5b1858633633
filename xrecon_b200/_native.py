"""ctypes binding of libxrecon_b200.so (the C ABI of include/xrecon_b200.h).

Only CUDA tensors are accepted: there is no CPU path.  A missing library or a
CPU tensor raises immediately.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_float, c_int, c_size_t, c_void_p
from pathlib import Path

import torch

from . import build as _build

OPS = {"A": 0, "AT": 1, "B": 2, "BT": 3, "BW": 4, "BWT": 5}
SINO_OUT = {"A", "BT", "BWT"}
DTYPES = {torch.float32: 0, torch.bfloat16: 1, torch.float16: 2}
SCAN_IDS = {"parallel": 0, "flat": 1, "arc": 2}


class Geom2d(ctypes.Structure):
    _fields_ = [("W", c_int), ("H", c_int), ("Nu", c_int), ("type", c_int),
                ("dx", c_float), ("dy", c_float), ("du", c_float), ("sod", c_float), ("sdd", c_float),
                ("shift_x", c_float), ("shift_y", c_float), ("shift_u", c_float)]


class Geom3d(ctypes.Structure):
    _fields_ = [("W", c_int), ("H", c_int), ("D", c_int), ("Nu", c_int), ("Nv", c_int), ("type", c_int),
                ("dx", c_float), ("dy", c_float), ("dz", c_float), ("du", c_float), ("dv", c_float),
                ("sod", c_float), ("sdd", c_float),
                ("shift_x", c_float), ("shift_y", c_float), ("shift_z", c_float),
                ("shift_u", c_float), ("shift_v", c_float)]


class HelicalOpts(ctypes.Structure):
    """xr_helical_opts: entries 18..23 of HelicalProjector3d's options."""
    _fields_ = [("view_mode", c_int), ("weight_mode", c_int), ("view_turns", c_float),
                ("halfscan_coef", c_float), ("tang_k", c_float), ("tang_blend", c_float)]


_lib = None


def library_path() -> Path:
    return _build.LIB


def lib():
    """Load the CUDA library, building it first when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not path.exists():
        _build.build()
    L = ctypes.CDLL(str(path))
    L.xr_dd2d_workspace_size.restype = c_size_t
    L.xr_dd2d_workspace_size.argtypes = [c_int, ctypes.POINTER(Geom2d), c_int, c_int]
    L.xr_dd3d_workspace_size.restype = c_size_t
    L.xr_dd3d_workspace_size.argtypes = [c_int, ctypes.POINTER(Geom3d), c_int, c_int]
    common = [c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_int, c_void_p, c_size_t, c_void_p]
    L.xr_dd2d.restype = c_int
    L.xr_dd2d.argtypes = [c_int, ctypes.POINTER(Geom2d)] + common
    L.xr_dd3d.restype = c_int
    L.xr_dd3d.argtypes = [c_int, ctypes.POINTER(Geom3d)] + common
    L.xr_dd2d_noalloc.restype = c_int
    L.xr_dd2d_noalloc.argtypes = [c_int, ctypes.POINTER(Geom2d), c_void_p, c_int, c_void_p, c_int,
                                  c_void_p, c_int, c_int, c_void_p]
    L.xr_fbp_filter.restype = c_int
    L.xr_fbp_filter.argtypes = [c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int,
                                c_void_p, c_void_p, c_void_p, c_void_p]
    L.xr_device_error.restype = c_int
    L.xr_device_error.argtypes = [ctypes.POINTER(ctypes.c_uint), c_int]
    L.xr_cell_plan.restype = c_int
    L.xr_cell_plan.argtypes = [ctypes.POINTER(Geom3d)] + [ctypes.POINTER(c_int)] * 5
    L.xr_pfx_stage_plan.restype = c_int
    L.xr_pfx_stage_plan.argtypes = [ctypes.POINTER(Geom3d)] + [ctypes.POINTER(c_int)] * 3
    L.xr_set_plain_kernels.restype = c_int
    L.xr_set_plain_kernels.argtypes = [c_int]
    L.xr_set_wait_limits.restype = c_int
    L.xr_set_wait_limits.argtypes = [ctypes.c_longlong, ctypes.c_longlong]
    L.xr_test_hooks.restype = c_int
    L.xr_test_hooks.argtypes = [ctypes.c_uint]
    L.xr_last_error.restype = ctypes.c_char_p
    for d, G in ((2, Geom2d), (3, Geom3d)):
        ws = getattr(L, f"xr_sysmat{d}d_workspace_size")
        ws.restype = c_size_t
        ws.argtypes = [ctypes.POINTER(G), c_int]
        fn = getattr(L, f"xr_sysmat{d}d")
        fn.restype = c_int
        fn.argtypes = [ctypes.POINTER(G), c_void_p, c_int] + [c_void_p] * 5 + [c_void_p, c_size_t, c_void_p]
    L.xr_helical3d_workspace_size.restype = c_size_t
    L.xr_helical3d_workspace_size.argtypes = [c_int, ctypes.POINTER(Geom3d), c_int, c_int]
    L.xr_helical3d.restype = c_int
    L.xr_helical3d.argtypes = [c_int, ctypes.POINTER(Geom3d), ctypes.POINTER(HelicalOpts), c_void_p, c_void_p,
                               c_void_p, c_void_p, c_int, c_int, c_void_p, c_size_t, c_void_p]
    L.xr_ctpd_load.restype = c_int
    L.xr_ctpd_load.argtypes = [ctypes.POINTER(ctypes.c_char_p)] + [c_int] * 6 + [c_void_p, c_void_p,
                                                                                 ctypes.POINTER(c_int)]
    L.xr_launch_count.restype = ctypes.c_ulonglong
    L.xr_launch_count.argtypes = []
    L.xr_version.restype = ctypes.c_char_p
    _lib = L
    return L


def _raise(rc: int, what: str):
    msg = lib().xr_last_error().decode(errors="replace")
    raise RuntimeError(f"{what} failed (status {rc}): {msg}")


def _f32(v) -> float:
    import numpy as np
    return float(np.float32(v))


def geom2d_from_values(vals) -> Geom2d:
    """From the 12 packed options of the reference (projector.py:106-110),
    field order of torch_binding.cpp:62-79."""
    v = [float(x) for x in vals]
    return Geom2d(W=int(v[0]), H=int(v[1]), Nu=int(v[2]), type=int(v[11]),
                  dx=v[3], dy=v[4], du=v[5], sod=v[6], sdd=v[7],
                  shift_x=v[8], shift_y=v[9], shift_u=v[10])


def geom3d_from_values(vals) -> Geom3d:
    """From the 18 packed options (projector3d.py:98-107), field order of
    torch_binding.cpp:82-124."""
    v = [float(x) for x in vals]
    return Geom3d(W=int(v[0]), H=int(v[1]), D=int(v[2]), Nu=int(v[3]), Nv=int(v[4]), type=int(v[17]),
                  dx=v[5], dy=v[6], dz=v[7], du=v[8], dv=v[9], sod=v[10], sdd=v[11],
                  shift_x=v[12], shift_y=v[13], shift_z=v[14], shift_u=v[15], shift_v=v[16])


def _check_cuda(name: str, t: torch.Tensor):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (xrecon_b200 has no CPU path)")


def _workspace(nbytes: int, device) -> torch.Tensor:
    # torch's caching allocator returns 512-byte aligned blocks.
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def _angles(angles: torch.Tensor, device) -> torch.Tensor:
    if angles.dim() != 1:
        raise RuntimeError(f"angles must be 1-D [V], got shape {tuple(angles.shape)}")
    return angles.to(device=device, dtype=torch.float32).contiguous()


def apply(dim: int, op: str, x: torch.Tensor, geom, angles: torch.Tensor,
          out_dtype: torch.dtype | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
    """Run one DD operator on a CUDA tensor; returns a new tensor."""
    _check_cuda("input", x)
    if x.dtype not in DTYPES:
        raise RuntimeError(f"input dtype {x.dtype} not supported (float32, bfloat16, float16)")
    if not x.is_contiguous():
        raise RuntimeError("Expected all tensors to be contiguous")
    dev = x.device
    ang = _angles(angles, dev)
    V = ang.numel()
    if dim == 2:
        if x.dim() != 4:
            raise RuntimeError(f"Expected 4-D input [B, C, ...], got {tuple(x.shape)}")
        if op in SINO_OUT:
            if tuple(x.shape[2:]) != (geom.H, geom.W):
                raise RuntimeError(f"Image shape {tuple(x.shape[2:])} does not match geometry {(geom.H, geom.W)}")
            shape = (x.shape[0], x.shape[1], V, geom.Nu)
        else:
            if tuple(x.shape[2:]) != (V, geom.Nu):
                raise RuntimeError(f"Sinogram shape {tuple(x.shape[2:])} does not match {(V, geom.Nu)}")
            shape = (x.shape[0], x.shape[1], geom.H, geom.W)
    else:
        if x.dim() != 5:
            raise RuntimeError(f"Expected 5-D input [B, C, ...], got {tuple(x.shape)}")
        if op in SINO_OUT:
            if tuple(x.shape[2:]) != (geom.D, geom.H, geom.W):
                raise RuntimeError("Image shape does not match 3D geometry")
            shape = (x.shape[0], x.shape[1], V, geom.Nv, geom.Nu)
        else:
            if tuple(x.shape[2:]) != (V, geom.Nv, geom.Nu):
                raise RuntimeError("Sinogram shape does not match 3D geometry")
            shape = (x.shape[0], x.shape[1], geom.D, geom.H, geom.W)
    odt = out_dtype or x.dtype
    if odt not in DTYPES:
        raise RuntimeError(f"output dtype {odt} not supported")
    if out is None:
        out = torch.empty(shape, dtype=odt, device=dev)
    elif tuple(out.shape) != shape or out.dtype != odt or not out.is_contiguous() or out.device != dev:
        raise RuntimeError("provided output tensor has the wrong shape, dtype, layout or device")
    nbatch = int(x.shape[0] * x.shape[1])
    if out.numel() == 0 or nbatch == 0:
        return out
    L = lib()
    with torch.cuda.device(dev):
        if dim == 2:
            nbytes = L.xr_dd2d_workspace_size(OPS[op], ctypes.byref(geom), nbatch, V)
            fn = L.xr_dd2d
        else:
            nbytes = L.xr_dd3d_workspace_size(OPS[op], ctypes.byref(geom), nbatch, V)
            fn = L.xr_dd3d
        ws = _workspace(nbytes, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = fn(OPS[op], ctypes.byref(geom), x.data_ptr(), DTYPES[x.dtype], out.data_ptr(), DTYPES[odt],
                ang.data_ptr(), nbatch, V, ws.data_ptr(), ws.numel(), stream)
    if rc != 0:
        _raise(rc, f"xr_dd{dim}d({op})")
    _after_op()
    return out


def helical_opts_from_values(vals) -> HelicalOpts:
    """Entries 18..23 of the packed helical options with the binding's
    defaults when absent (torch_binding.cpp:103-108)."""
    v = [float(x) for x in vals]
    get = (lambda i, d: v[i] if len(v) > i else d)
    return HelicalOpts(view_mode=int(get(18, 2.0)), weight_mode=int(get(19, 0.0)), view_turns=get(20, 0.0),
                       halfscan_coef=get(21, 1.0), tang_k=get(22, 5.0), tang_blend=get(23, 0.0))


def helical(op: str, x: torch.Tensor, geom: Geom3d, hopts: HelicalOpts, angles: torch.Tensor,
            source_pos: torch.Tensor) -> torch.Tensor:
    """Run one helical operator (float32) on a CUDA tensor; returns a new tensor."""
    _check_cuda("input", x)
    dev = x.device
    if x.dtype != torch.float32:
        raise RuntimeError("Helical 3D tensors must be float32")
    if x.dim() != 5 or not x.is_contiguous():
        raise RuntimeError("input must be a contiguous 5-D tensor")
    ang = _angles(angles, dev)
    V = ang.numel()
    sp = source_pos.to(device=dev, dtype=torch.float32).contiguous()
    if tuple(sp.shape) != (4, V):
        raise RuntimeError("source_pos must have shape [4, num_view]")
    if op in SINO_OUT:
        shape = (x.shape[0], x.shape[1], V, geom.Nv, geom.Nu)
    else:
        shape = (x.shape[0], x.shape[1], geom.D, geom.H, geom.W)
    nbatch = int(x.shape[0] * x.shape[1])
    if V == 0 or nbatch == 0 or x.numel() == 0:
        return torch.zeros(shape, dtype=torch.float32, device=dev)
    out = torch.empty(shape, dtype=torch.float32, device=dev)
    L = lib()
    with torch.cuda.device(dev):
        nbytes = L.xr_helical3d_workspace_size(OPS[op], ctypes.byref(geom), nbatch, V)
        ws = _workspace(nbytes, dev)
        rc = L.xr_helical3d(OPS[op], ctypes.byref(geom), ctypes.byref(hopts), x.data_ptr(), out.data_ptr(),
                            ang.data_ptr(), sp.data_ptr(), nbatch, V, ws.data_ptr(), ws.numel(),
                            torch.cuda.current_stream(dev).cuda_stream)
    if rc != 0:
        _raise(rc, f"xr_helical3d({op})")
    _after_op()
    return out


def fbp_filter(sino: torch.Tensor, nview: int, rows_per_view: int, cosw: torch.Tensor | None,
               filt: torch.Tensor, parker: torch.Tensor | None) -> torch.Tensor:
    """Fused cosine weight x Parker weight x spatial filter correlation along u."""
    _check_cuda("sino", sino)
    if sino.dtype not in DTYPES or not sino.is_contiguous():
        raise RuntimeError("sinogram must be a contiguous float32/bfloat16/float16 CUDA tensor")
    dev = sino.device
    Nu = sino.shape[-1]
    nrows = sino.numel() // Nu if Nu else 0
    out = torch.empty(sino.shape, dtype=torch.float32, device=dev)
    if nrows == 0:
        return out
    f = filt.to(device=dev, dtype=torch.float32).contiguous().reshape(-1)
    if f.numel() != 2 * Nu - 1:
        raise RuntimeError(f"filter must have 2*Nu-1 = {2 * Nu - 1} taps, got {f.numel()}")
    cw = None if cosw is None else cosw.to(device=dev, dtype=torch.float32).contiguous().reshape(-1)
    pk = None if parker is None else parker.to(device=dev, dtype=torch.float32).contiguous().reshape(-1)
    with torch.cuda.device(dev):
        rc = lib().xr_fbp_filter(sino.data_ptr(), DTYPES[sino.dtype], out.data_ptr(), nrows, Nu, nview,
                                 rows_per_view, None if cw is None else cw.data_ptr(), f.data_ptr(),
                                 None if pk is None else pk.data_ptr(),
                                 torch.cuda.current_stream(dev).cuda_stream)
    if rc != 0:
        _raise(rc, "xr_fbp_filter")
    return out


def system_matrix(dim: int, geom, angles: torch.Tensor, device) -> torch.Tensor:
    """Sparse COO matrix of the projection (rows: view, detector row, column;
    columns: voxels), built on ``device`` in two passes (count, scan, fill)
    and coalesced, as the reference's system_matrix2d/3d returns it."""
    L = lib()
    dev = torch.device(device)
    ang = _angles(angles, dev)
    V = ang.numel()
    if V == 0:
        raise RuntimeError("system matrix needs at least one view")
    Nv = geom.Nv if dim == 3 else 1
    D = geom.D if dim == 3 else 1
    ncell = V * Nv * geom.Nu
    with torch.cuda.device(dev):
        nbytes = getattr(L, f"xr_sysmat{dim}d_workspace_size")(ctypes.byref(geom), V)
        ws = _workspace(nbytes, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        fn = getattr(L, f"xr_sysmat{dim}d")
        counts = torch.empty(ncell, dtype=torch.int64, device=dev)
        rc = fn(ctypes.byref(geom), ang.data_ptr(), V, None, counts.data_ptr(), None, None, None,
                ws.data_ptr(), ws.numel(), stream)
        if rc != 0:
            _raise(rc, f"xr_sysmat{dim}d (count)")
        ends = torch.cumsum(counts, 0)
        nnz = int(ends[-1].item())
        offsets = ends - counts
        rows = torch.empty(nnz, dtype=torch.int64, device=dev)
        cols = torch.empty(nnz, dtype=torch.int64, device=dev)
        vals = torch.empty(nnz, dtype=torch.float32, device=dev)
        if nnz:
            rc = fn(ctypes.byref(geom), ang.data_ptr(), V, offsets.data_ptr(), counts.data_ptr(), rows.data_ptr(),
                    cols.data_ptr(), vals.data_ptr(), ws.data_ptr(), ws.numel(), stream)
            if rc != 0:
                _raise(rc, f"xr_sysmat{dim}d (fill)")
        shape = (V * Nv * geom.Nu, D * geom.H * geom.W)
        return torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, shape, check_invariants=False).coalesce()


def device_error(clear: bool = True) -> int:
    """Device-wide error word of the current device (0 = no kernel reported a
    problem; bit 0: a TMA wait of the projection kernel gave up, bit 1: a grid
    barrier of the ragged kernel gave up).  Synchronous."""
    code = ctypes.c_uint(0)
    rc = lib().xr_device_error(ctypes.byref(code), int(clear))
    if rc != 0:
        _raise(rc, "xr_device_error")
    return int(code.value)


def check_device_error() -> None:
    """Raise RuntimeError (and clear the word) when a kernel of this library
    reported a bounded wait that gave up since the last check: the outputs of
    that launch are not valid.  Synchronous; the operators do not call it
    themselves unless the environment sets XRECON_B200_CHECK=1."""
    code = device_error(clear=True)
    if code:
        what = []
        if code & 1:
            what.append("a TMA transfer wait of the projection kernel gave up")
        if code & 2:
            what.append("a grid barrier of the ragged batch kernel gave up")
        raise RuntimeError(f"xrecon_b200 device error {code:#x}: " + "; ".join(what or ["unknown code"]))


_CHECK_EACH = os.environ.get("XRECON_B200_CHECK", "") not in ("", "0")


def _after_op() -> None:
    if _CHECK_EACH:
        check_device_error()


def set_wait_limits(tma_polls: int = 0, barrier_polls: int = 0) -> None:
    """Poll limits of the bounded waits on the current device (<= 0: the
    defaults, 2^20 TMA polls of at most ~1 us and 2^22 barrier polls of ~128 ns)."""
    rc = lib().xr_set_wait_limits(int(tma_polls), int(barrier_polls))
    if rc != 0:
        _raise(rc, "xr_set_wait_limits")


def test_hooks(bits: int) -> None:
    """Failure injection for the bounded waits (testing aid; 0 = off): bit 0
    stalls the projection kernel's TMA copies, bit 1 makes the ragged grid
    barriers wait for one block too many."""
    rc = lib().xr_test_hooks(int(bits))
    if rc != 0:
        _raise(rc, "xr_test_hooks")


def cell_plan(geom: Geom3d) -> dict:
    """Staging plan of the 3D projection kernel (TMA box size) for a geometry."""
    vals = [c_int(0) for _ in range(5)]
    rc = lib().xr_cell_plan(ctypes.byref(geom), *[ctypes.byref(v) for v in vals])
    if rc != 0:
        _raise(rc, "xr_cell_plan")
    return dict(ok=bool(vals[0].value), box_pixels=vals[1].value, box_z=vals[2].value,
                rows_per_thread=vals[3].value, fine=bool(vals[4].value))


def pfx_stage_plan(geom: Geom3d) -> dict:
    """Staging plan of the 3D prefix backprojection (table box size) for a geometry."""
    vals = [c_int(0) for _ in range(3)]
    rc = lib().xr_pfx_stage_plan(ctypes.byref(geom), *[ctypes.byref(v) for v in vals])
    if rc != 0:
        _raise(rc, "xr_pfx_stage_plan")
    return dict(ok=bool(vals[0].value), box_cols=vals[1].value, box_rows=vals[2].value)


def set_plain_kernels(on: bool) -> None:
    """Route operators through the plain (non-TMA) kernels (testing aid)."""
    lib().xr_set_plain_kernels(int(bool(on)))


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(lib().xr_launch_count())


def version() -> str:
    return lib().xr_version().decode()
