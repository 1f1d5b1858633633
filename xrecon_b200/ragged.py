"""Ragged batches of 2D reconstructions in one persistent launch.

``RaggedFBP2d`` takes a list of ``Projector2d`` instances with their angles
(any mix of image sizes, view counts, detectors and geometries), lays their
images, sinograms and reconstructions back to back on the device, and runs
projection followed by FBP for all of them in one persistent cooperative
kernel (``xr_ragged2d_run``).  The tile shapes of the projection and
backprojection phases are picked by a small autotuner that times the
candidates on the batch itself (cached per batch signature), and the launch
is captured in a CUDA graph, so a call is one graph replay.

The FBP follows ``Projector2d.filtered_backprojection`` for a full scan
without Parker weighting (projector.py:176-206 of the reference): the same
cosine weight and filter taps, the weighted backprojection, and the scale
mean|d beta| / 2.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import torch

from . import _native
from .projector import Projector2d, mean_angle_step

_c_ll = ctypes.c_longlong


class RaggedInstance(ctypes.Structure):
    _fields_ = [("geom", _native.Geom2d), ("nview", ctypes.c_int),
                ("img_offset", _c_ll), ("sino_offset", _c_ll), ("ang_offset", _c_ll),
                ("filt_offset", _c_ll), ("cosw_offset", _c_ll), ("scale", ctypes.c_float)]


def _lib():
    L = _native.lib()
    if not getattr(L, "_ragged_ready", False):
        L.xr_ragged2d_plan_create.restype = ctypes.c_int
        L.xr_ragged2d_plan_create.argtypes = [ctypes.POINTER(RaggedInstance), ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]
        L.xr_ragged2d_plan_bind.restype = ctypes.c_int
        L.xr_ragged2d_plan_bind.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 7 + [ctypes.c_size_t]
        L.xr_ragged2d_run.restype = ctypes.c_int
        L.xr_ragged2d_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.xr_ragged2d_plan_info.restype = ctypes.c_int
        L.xr_ragged2d_plan_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]
        L.xr_ragged2d_plan_destroy.restype = None
        L.xr_ragged2d_plan_destroy.argtypes = [ctypes.c_void_p]
        L._ragged_ready = True
    return L


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed (status {rc}): {_native.lib().xr_last_error().decode()}")


_TUNED: dict = {}  # batch signature -> (a_cols_log2, view_split_log2)


class RaggedFBP2d:
    """Projection + FBP of a ragged batch of 2D instances, one launch per call.

    ``projectors[i]`` is a ``Projector2d`` and ``angles[i]`` its view angles
    (radians, 1-D).  ``__call__(images)`` takes a list of [H_i, W_i] (or
    [1, 1, H_i, W_i]) float32 CUDA tensors and returns (sinograms,
    reconstructions), each a list of views into the batch buffers.

    Each reconstruction is ``projectors[i].filtered_backprojection`` of its
    sinogram with that method's defaults: the projector's own filter and
    cosine weight, no Parker weights, and the redundant-scan factor 1/2 on
    the mean angular step.  Short scans that need Parker weights go through
    ``Projector2d.filtered_backprojection(..., parker=True)`` instead.
    """

    def __init__(self, projectors: Sequence[Projector2d], angles: Sequence[torch.Tensor],
                 device: Optional[torch.device] = None, autotune: bool = True, graph: bool = True):
        if len(projectors) != len(angles) or not projectors:
            raise ValueError("need one angle vector per projector")
        self.device = torch.device(device or "cuda")
        L = _lib()
        inst = (RaggedInstance * len(projectors))()
        self.shapes: List[Tuple[int, int, int, int]] = []
        img_off = sino_off = ang_off = filt_off = cosw_off = 0
        filts, cosws, angs = [], [], []
        for i, (P, a) in enumerate(zip(projectors, angles)):
            a = a.detach().to(torch.float32).reshape(-1).cpu()
            W, H = P.image_size
            Nu = P.num_det
            V = a.numel()
            g = _native.geom2d_from_values(P.options.detach().cpu().tolist())
            inst[i].geom = g
            inst[i].nview = V
            inst[i].img_offset, inst[i].sino_offset, inst[i].ang_offset = img_off, sino_off, ang_off
            inst[i].filt_offset, inst[i].cosw_offset = filt_off, cosw_off
            inst[i].scale = float(mean_angle_step(a)) / 2.0
            self.shapes.append((H, W, V, Nu))
            filts.append(P.filter.detach().reshape(-1).to(torch.float32).cpu())
            cosws.append(P.weight.detach().reshape(-1).to(torch.float32).cpu())
            angs.append(a)
            img_off += H * W
            sino_off += V * Nu
            ang_off += V
            filt_off += 2 * Nu - 1
            cosw_off += Nu
        self._inst = inst
        plan = ctypes.c_void_p()
        nbytes = ctypes.c_size_t()
        _check(L.xr_ragged2d_plan_create(inst, len(projectors), ctypes.byref(plan), ctypes.byref(nbytes)),
               "xr_ragged2d_plan_create")
        self._plan = plan
        dev = self.device
        with torch.cuda.device(dev):
            self.images = torch.zeros(img_off, dtype=torch.float32, device=dev)
            self.recon = torch.zeros(img_off, dtype=torch.float32, device=dev)
            self.sino = torch.zeros(sino_off, dtype=torch.float32, device=dev)
            self.angles = torch.cat(angs).to(dev)
            self.filt = torch.cat(filts).to(dev)
            self.cosw = torch.cat(cosws).to(dev)
            self.workspace = torch.empty(max(int(nbytes.value), 256), dtype=torch.uint8, device=dev)
            _check(L.xr_ragged2d_plan_bind(plan, self.images.data_ptr(), self.sino.data_ptr(), self.recon.data_ptr(),
                                           self.angles.data_ptr(), self.filt.data_ptr(), self.cosw.data_ptr(),
                                           self.workspace.data_ptr(), self.workspace.numel()),
                   "xr_ragged2d_plan_bind")
        self.config = (2, 0)
        self.signature = tuple((tuple(s), round(float(inst[i].geom.du), 6), round(float(inst[i].geom.sod), 3),
                                int(inst[i].geom.type)) for i, s in enumerate(self.shapes))
        self._graph = None
        if autotune:
            self.autotune()
        if graph:
            self.capture()

    # ------------------------------------------------------------ launches
    def launch(self, project: bool = True, config: Optional[Tuple[int, int]] = None) -> None:
        """One persistent launch on the current stream (eager)."""
        a, v = config or self.config
        with torch.cuda.device(self.device):
            _check(_lib().xr_ragged2d_run(self._plan, int(bool(project)), a, v,
                                          torch.cuda.current_stream(self.device).cuda_stream), "xr_ragged2d_run")

    def info(self) -> dict:
        grid = ctypes.c_int()
        tiles = (ctypes.c_int * 10)()
        _check(_lib().xr_ragged2d_plan_info(self._plan, ctypes.byref(grid), tiles), "xr_ragged2d_plan_info")
        return {"grid": grid.value, "tiles": list(tiles), "config": self.config}

    def autotune(self, reps: int = 3) -> Tuple[int, int]:
        """Time every (projection columns, view split) pair on this batch and
        keep the fastest; results are cached per batch signature."""
        if self.signature in _TUNED:
            self.config = _TUNED[self.signature]
            return self.config
        best = None
        with torch.cuda.device(self.device):
            for a in range(4):
                for v in range(4):
                    self.launch(True, (a, v))  # warm-up
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(reps):
                        self.launch(True, (a, v))
                    e1.record()
                    torch.cuda.synchronize()
                    t = e0.elapsed_time(e1) / reps
                    if best is None or t < best[0]:
                        best = (t, (a, v))
        self.config = best[1]
        self.tuned_ms = best[0]
        _TUNED[self.signature] = self.config
        return self.config

    def capture(self) -> None:
        """Capture the launch (projection + FBP) in a CUDA graph."""
        with torch.cuda.device(self.device):
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                self.launch(True)  # warm-up outside the capture
            torch.cuda.current_stream(self.device).wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self.launch(True)
            self._graph = g

    def run(self) -> None:
        """Projection + FBP of the images currently in ``self.images``."""
        if self._graph is not None:
            self._graph.replay()
        else:
            self.launch(True)

    # ------------------------------------------------------------- access
    def set_images(self, images: Sequence[torch.Tensor]) -> None:
        off = 0
        for (H, W, _, _), im in zip(self.shapes, images):
            self.images[off:off + H * W].copy_(im.reshape(-1), non_blocking=True)
            off += H * W

    def sinograms(self) -> List[torch.Tensor]:
        out, off = [], 0
        for H, W, V, Nu in self.shapes:
            out.append(self.sino[off:off + V * Nu].view(1, 1, V, Nu))
            off += V * Nu
        return out

    def reconstructions(self) -> List[torch.Tensor]:
        out, off = [], 0
        for H, W, V, Nu in self.shapes:
            out.append(self.recon[off:off + H * W].view(1, 1, H, W))
            off += H * W
        return out

    def __call__(self, images: Sequence[torch.Tensor]):
        self.set_images(images)
        self.run()
        return self.sinograms(), self.reconstructions()

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _lib().xr_ragged2d_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None
