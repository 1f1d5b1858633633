#!/usr/bin/env python
"""Benchmark of the distance-driven projector path.

Workload (the headline configuration): cone-beam flat detector, volume
512x512x256 at 0.75 mm (random-ellipsoid phantom, densities in [0, 1]),
1440 views over 2*pi, detector 1024x256 at 0.8 mm, SOD 595 mm, SDD 1085 mm.
One step = forward projection A followed by backprojection B of the
resulting sinogram, FP32, inputs resident in HBM (both larger than L2).

    value = B*C*Nx*Ny*Nz*V / (t_A + t_B) / 1e9      [Gvoxel-views/s]

summed over ranks (one independent reconstruction per GPU, weak scaling).
The roofline denominator is the measured HBM copy bandwidth; the algorithmic
bytes of one operator application are V*(Nvox + Nu*Nv)*4 (each view streams
the volume and its own projection once).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DD fwd+back Gvoxel-views/s (batched/BF16 vs plain FP32 @1e-3 rel); %HBM peak"
UNIT = "Gvoxel-views/s"
WL = dict(W=512, H=512, D=256, Nu=1024, Nv=256, V=1440, dx=0.75, du=0.8, sod=595.0, sdd=1085.0)
WORKLOAD_NAME = "cone-flat 512x512x256 vol, 1440 views, 1024x256 det, fwd A + back B"
FALLBACK_HBM = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


def nvox(wl=WL):
    return wl["W"] * wl["H"] * wl["D"]


def algo_bytes_op(wl=WL, s=4):
    return wl["V"] * (nvox(wl) + wl["Nu"] * wl["Nv"]) * s


def make_projector():
    import xrecon_b200 as xr
    return xr.Projector3d(xr.Volume3d((WL["W"], WL["H"], WL["D"]), WL["dx"]),
                          xr.ConeBeam3d(xr.Detector3d((WL["Nu"], WL["Nv"]), WL["du"]), WL["sod"], WL["sdd"], "flat"))


def angles_np(nviews=None, contiguous=False):
    """The workload's views, uniform over 2 pi; with ``nviews`` an evenly
    strided subset, or with ``contiguous`` the first ``nviews`` neighbouring
    views (profiling cases)."""
    import numpy as np
    a = (np.arange(WL["V"]) * (2 * np.pi / WL["V"])).astype(np.float32)
    if nviews is None or nviews >= WL["V"]:
        return a
    if contiguous:
        return a[:nviews].copy()
    return a[:: WL["V"] // nviews][:nviews].copy()


def ragged_c4_batch(seed: int = 4, count: int = 64):
    """The ragged 2D fan-arc batch: per instance, image size N in {128, 192,
    256, 384, 512} (pixel 512/N mm), views uniform in [180, 1440] over 2 pi,
    detector cells uniform in [192, 736] of 1.0-2.0 mm, SOD uniform in
    [400, 600] mm, SDD = 2 SOD; random-ellipse phantoms.  Returns
    (projectors, angles, images) with images as float32 numpy arrays."""
    import numpy as np
    from xrecon_b200 import geometry as G
    from xrecon_b200.phantom import create_phantom2d, random_ellipses2d
    from xrecon_b200.projector import Projector2d
    rng = np.random.default_rng(seed)
    projectors, angles, images = [], [], []
    for i in range(count):
        N = int(rng.choice([128, 192, 256, 384, 512]))
        V = int(rng.integers(180, 1441))
        Nu = int(rng.integers(192, 737))
        du = float(rng.uniform(1.0, 2.0))
        sod = float(rng.uniform(400.0, 600.0))
        geo = G.FanBeam2d(G.Detector2d(Nu, du), sod, 2.0 * sod, "arc")
        projectors.append(Projector2d(G.Volume2d(N, 512.0 / N), geo))
        angles.append((np.arange(V) * (2 * np.pi / V)).astype(np.float32))
        images.append(create_phantom2d((N, N), random_ellipses2d(10, seed=1000 * seed + i, n=N)))
    return projectors, angles, images


# ---------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = Path(f"/tmp/xr_bench_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.idx), "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------- CPU reference

_CPU_VOL = None


def cpu_volume():
    """The seeded phantom of rank 0, rasterised with torch on the host."""
    global _CPU_VOL
    if _CPU_VOL is None:
        from xrecon_b200.phantom import ellipsoid_volume_torch, random_ellipsoids3d
        v = ellipsoid_volume_torch((WL["D"], WL["H"], WL["W"]), random_ellipsoids3d(20, seed=0, density=(0.0, 1.0)),
                                   "cpu")
        _CPU_VOL = v.numpy()[None, None]
    return _CPU_VOL


def cpu_reference_sample(nviews: int = 4, vol=None):
    """The reference's own CPU operators (oracle/_ref, std::thread x
    hardware_concurrency) on `nviews` views of the workload: A then B."""
    from oracle import refcpu
    if not refcpu.available():
        return None
    P = make_projector()
    opts = P.options.numpy()
    vol = cpu_volume() if vol is None else vol
    ang = angles_np()[:: WL["V"] // nviews][:nviews].copy()
    t0 = time.perf_counter()
    sino = refcpu.dd3d("A", vol, opts, ang)
    t1 = time.perf_counter()
    refcpu.dd3d("B", sino, opts, ang)
    t2 = time.perf_counter()
    cores = os.cpu_count() or 1
    value = nvox() * nviews / (t2 - t0) / 1e9
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{nviews} of {WL['V']} views of the workload (A {t1 - t0:.1f}s + B {t2 - t1:.1f}s)",
            "seconds": t2 - t0}


def helical_reference_measure(reps: int = 1):
    """The reference's own helical CUDA kernels (helical_arc3d.cu built
    unchanged into oracle/_ref by oracle/build_oracle.py) on the HEL workload:
    device times of A, B and Bw, the same operators helical_measure times on
    this library.  Outputs carry a zero guard band of one plane on both sides
    (the reference's scatter kernels index them from FP32 guesses)."""
    import ctypes
    import numpy as np
    import torch
    from oracle import build_oracle
    so = build_oracle.REF_HELICAL_SO
    if not so.exists() or not torch.cuda.is_available():
        return {"unavailable": "reference helical library oracle/_ref not built or no GPU"}
    lib = ctypes.CDLL(str(so))
    lib.xr_ref_helical.restype = ctypes.c_int
    lib.xr_ref_helical.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_float)] + [ctypes.c_void_p] * 4 + \
                                  [ctypes.c_int, ctypes.c_int]
    dev = torch.device("cuda:0")
    P, ang = helical_projector(dev)
    opts = (ctypes.c_float * 24)(*P.options.cpu().tolist())
    sp = P.source_position(ang).contiguous()
    h = HEL
    V = ang.numel()
    nvox, ncell = h["W"] * h["H"] * h["D"], V * h["Nv"] * h["Nu"]
    gi, gs = h["W"] * h["H"], h["Nv"] * h["Nu"]
    g = torch.Generator(device=dev).manual_seed(3)
    img = torch.zeros(nvox + 2 * gi, device=dev)
    sino = torch.zeros(ncell + 2 * gs, device=dev)
    img[gi:gi + nvox] = torch.rand(nvox, device=dev, generator=g)
    ip, sp_ = img.data_ptr() + 4 * gi, sino.data_ptr() + 4 * gs
    out = {}
    for op, key, zero_img in ((0, "A_ms", False), (2, "B_ms", True), (4, "Bw_ms", True)):
        ts = []
        for i in range(reps + 1):
            if zero_img:
                img.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            rc = lib.xr_ref_helical(op, opts, ip, sp_, ang.data_ptr(), sp.data_ptr(), 1, V)
            e1.record()
            torch.cuda.synchronize()
            if rc != 0:
                return {"unavailable": f"reference helical op {op} returned CUDA error {rc}"}
            if i > 0:
                ts.append(e0.elapsed_time(e1))
        out[key] = sum(ts) / len(ts)
    out["guard_ok"] = bool(img[:gi].abs().max() == 0 and img[gi + nvox:].abs().max() == 0 and
                           sino[:gs].abs().max() == 0 and sino[gs + ncell:].abs().max() == 0)
    out["views"] = int(V)
    del img, sino
    torch.cuda.empty_cache()
    return out


def run_reference_arm(args, rank: int):
    if rank != 0:
        return 0
    nviews = 2
    samples = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_sample(nviews)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU library oracle/_ref not built"}))
            return 0
        if i >= args.warmup:
            samples.append(r)
    t = sum(s["seconds"] for s in samples) / len(samples)
    value = nvox() * nviews / t / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random ellipsoids)",
        "config": {"workload": WORKLOAD_NAME, "step": f"A+B on {nviews} views (bounded CPU sample)"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": samples[0]["cores"], "kind": "reference",
                         "sample": samples[0]["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_helical:
        line["helical_arc_512x512x128_736x64_5x1152views"] = helical_reference_measure()
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm

def operator_times(P, vol, ang, nv, reps: int = 2):
    """Every operator and the FDK on the same workload (FP32), each timed
    alone with CUDA events: ms per application and Gvoxel-views/s."""
    import torch
    sino = P.projection(vol, ang)
    ops = {
        "projection_t (A^T)": lambda: P.projection_t(sino, ang),
        "backprojection_weighted (Bw)": lambda: P.backprojection_weighted(sino, ang),
        "backprojection_t (B^T)": lambda: P.backprojection_t(vol, ang),
        "backprojection_weighted_t (Bw^T)": lambda: P.backprojection_weighted_t(vol, ang),
        "filtered_backprojection (FDK)": lambda: P.filtered_backprojection(sino, ang),
    }
    out = {}
    for name, fn in ops.items():
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": ms, "gvoxel_views_per_s": nvox() * nv / (ms / 1e3) / 1e9}
    del sino
    return out


def sysmat_measure(dev, reps: int = 3):
    """Sparse projection-matrix export (count, scan, fill, coalesce) of the
    2D fan-flat geometry: 256x256 image of 1 mm, 720 views over 2 pi, 256
    cells of 2 mm, SOD 500, SDD 1000."""
    import numpy as np
    import torch
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector2d
    P = Projector2d(G.Volume2d(256, 1.0), G.FanBeam2d(G.Detector2d(256, 2.0), 500.0, 1000.0, "flat")).to(dev)
    ang = torch.from_numpy((np.arange(720) * (2 * np.pi / 720)).astype(np.float32)).to(dev)
    M = P.system_matrix(ang)
    nnz = M._nnz()
    del M
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        M = P.system_matrix(ang)
        del M
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return {"nnz": nnz, "ms": ms, "gnnz_per_s": nnz / (ms / 1e3) / 1e9}


def rebin_measure(P, vol, ang, reps: int = 3):
    """Fan -> parallel rebinning of the workload's sinogram (1440 views,
    256 rows, 1024 flat columns of 0.8 mm at SDD, i.e. 0.4387 mm at the
    isocentre) to 1024 parallel bins: this library's kernel, the same pass
    fused with a ramp filter, and torch.nn.functional.grid_sample on the
    same grid (the call the reference's rebinning makes)."""
    import torch
    import torch.nn.functional as F
    from xrecon_b200.filters import filter_generate
    from xrecon_b200.rebin import fan_to_parallel_rebin, rebin_grid
    sino = P.projection(vol, ang)
    du_iso = WL["du"] * WL["sod"] / WL["sdd"]
    args = (WL["sod"], du_iso, 0.0, "flat")

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    _, _, t = fan_to_parallel_rebin(sino, ang, *args)
    filt = filter_generate(WL["Nu"], float(t[1] - t[0]), "ramp", torch.float32).to(sino.device)
    ms = timed(lambda: fan_to_parallel_rebin(sino, ang, *args))
    ms_fused = timed(lambda: fan_to_parallel_rebin(sino, ang, *args, filt=filt))
    grid, _ = rebin_grid(ang, WL["Nu"], WL["sod"], du_iso, 0.0, "flat", ang, WL["Nu"], None, 0.0)
    src = sino.permute(0, 1, 3, 2, 4).reshape(WL["Nv"], 1, ang.numel(), WL["Nu"])
    g4 = grid[None].expand(WL["Nv"], -1, -1, -1)
    ms_torch = timed(lambda: F.grid_sample(src, g4, mode="bilinear", padding_mode="zeros", align_corners=True))
    del sino, src
    return {"ms": ms, "ms_fused_with_ramp_filter": ms_fused, "torch_grid_sample_ms": ms_torch,
            "samples": ang.numel() * WL["Nv"] * WL["Nu"]}


HEL = dict(W=512, H=512, D=128, dx=0.7, dz=0.8, Nu=736, Nv=64, du=1.2858, dv=1.0947, sod=595.0, sdd=1085.6,
           views_per_turn=1152, turns=5, pitch=30.7)


def helical_projector(dev, turns=None):
    """Helical scan of a 512 x 512 x 128 volume (0.7 x 0.7 x 0.8 mm) on a
    736 x 64 arc detector (1.2858 x 1.0947 mm cells at SDD 1085.6 mm, SOD
    595 mm), 1152 views per turn over 5 turns, 30.7 mm rise per turn
    (pitch 0.8 of the 38.4 mm collimation), one-turn view windows."""
    from xrecon_b200 import HelicalProjector3d
    h = dict(HEL, turns=turns or HEL["turns"])
    z_span = h["turns"] * h["pitch"]
    P = HelicalProjector3d((h["W"], h["H"], h["D"]), (h["Nu"], h["Nv"]), (h["dx"], h["dx"], h["dz"]),
                           (h["du"], h["dv"]), h["sod"], h["sdd"], pitch=h["pitch"], z0=-0.5 * z_span).to(dev)
    V = h["views_per_turn"] * h["turns"]
    import numpy as np
    import torch
    ang = torch.from_numpy((np.arange(V) * (2 * np.pi / h["views_per_turn"])).astype(np.float32)).to(dev)
    return P, ang


def helical_measure(dev, reps: int = 2, turns=None):
    """Per-operator device times of the helical projector (HEL workload;
    ``turns`` fewer turns for profiling captures); throughput in voxel-views
    per second counts each voxel against the views of one turn (the views
    whose source z is near the voxel's)."""
    import torch
    P, ang = helical_projector(dev, turns)
    h = HEL
    g = torch.Generator(device=dev).manual_seed(3)
    vol = torch.rand((1, 1, h["D"], h["H"], h["W"]), device=dev, generator=g)
    sino = P.projection(vol, ang)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    with torch.no_grad():
        out["A_ms"] = timed(lambda: P.projection(vol, ang))
        out["B_ms"] = timed(lambda: P.backprojection(sino, ang))
        out["Bw_ms"] = timed(lambda: P.backprojection_weighted(sino, ang))
        out["fdk_ms"] = timed(lambda: P.filtered_backprojection(sino, ang))
        out["BwT_ms"] = timed(lambda: P.backprojection_weighted_t(vol, ang))
    nvox = h["W"] * h["H"] * h["D"]
    out["gvoxel_views_per_turn_per_s_fdk"] = nvox * h["views_per_turn"] / (out["fdk_ms"] / 1e3) / 1e9
    out["views"] = int(ang.numel())
    del sino, vol
    torch.cuda.empty_cache()
    return out


def ragged_measure(dev, reps: int = 5):
    """The 64-instance ragged fan-arc batch: projection + FBP of every
    instance as one autotuned persistent launch replayed from a CUDA graph,
    next to the same work as a loop of per-instance Projector2d calls."""
    import torch
    from xrecon_b200.ragged import RaggedFBP2d
    projectors, angles, images = ragged_c4_batch()
    angs = [torch.from_numpy(a) for a in angles]
    R = RaggedFBP2d(projectors, angs, device=dev)
    imgs = [torch.from_numpy(im).to(dev) for im in images]
    R.set_images(imgs)
    R.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        R.run()
    e1.record()
    torch.cuda.synchronize()
    t_graph = e0.elapsed_time(e1) / reps / 1e3
    Ps = [P.to(dev) for P in projectors]
    dang = [a.to(dev) for a in angs]
    xs = [im[None, None] for im in imgs]

    def loop():
        for P, a, x in zip(Ps, dang, xs):
            P.filtered_backprojection(P.projection(x, a), a)

    loop()
    torch.cuda.synchronize()
    e0.record()
    loop()
    e1.record()
    torch.cuda.synchronize()
    t_loop = e0.elapsed_time(e1) / 1e3
    work = sum(P.image_size[0] * P.image_size[1] * a.numel() for P, a in zip(projectors, angs))
    return {"instances": len(projectors), "value": work / t_graph / 1e9, "unit": "Gpixel-views/s (A + FBP)",
            "ms": t_graph * 1e3, "per_instance_loop_ms": t_loop * 1e3,
            "tile_config": {"a_cols": 32 << R.config[0], "view_split": 1 << R.config[1]}}


# --------------------------------------------- the other baseline configs

def _timed_ms(fn, reps: int = 3) -> float:
    """Device time of fn() per call: CUDA events on the current stream,
    after one untimed call."""
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _cpu_filter_rows(sino_np, weight, filt):
    """The reference's FBP/FDK filter step on the host: cosine weight, then
    torch.nn.functional.conv2d of every detector row with the 2 Nu - 1 taps
    and Nu - 1 zero padding (projector.py:196-202, projector3d.py:185-191)."""
    import torch
    import torch.nn.functional as F
    x = torch.from_numpy(sino_np) * torch.as_tensor(weight).reshape(-1)
    Nu = x.shape[-1]
    rows = x.reshape(-1, 1, 1, Nu)
    return F.conv2d(rows, torch.as_tensor(filt).reshape(1, 1, 1, -1), padding=(0, Nu - 1)).reshape(x.shape).numpy()


def config_c1(dev, cpu: bool):
    """2D fan-flat 256x256 (1 mm) Shepp-Logan + 10 seeded ellipses, 720
    views over 2 pi, 256 cells of 2 mm, SOD 500, SDD 1000: projection, then
    ramp FBP.  value = 256^2 * 720 / (t_A + t_FBP)."""
    import numpy as np
    import torch
    from xrecon_b200 import geometry as G
    from xrecon_b200.phantom import shepp_logan_plus_ellipses2d
    from xrecon_b200.projector import Projector2d
    P = Projector2d(G.Volume2d(256, 1.0), G.FanBeam2d(G.Detector2d(256, 2.0), 500.0, 1000.0, "flat")).to(dev)
    img = shepp_logan_plus_ellipses2d(256, 10, seed=1).astype(np.float32)
    ang_np = (np.arange(720) * (2 * np.pi / 720)).astype(np.float32)
    x = torch.from_numpy(img)[None, None].to(dev)
    a = torch.from_numpy(ang_np).to(dev)
    sino = P.projection(x, a)
    t_a = _timed_ms(lambda: P.projection(x, a), 10)
    t_f = _timed_ms(lambda: P.filtered_backprojection(sino, a), 10)
    work = 256 * 256 * 720
    out = {"workload": "2D fan-flat 256x256, 720 views, 256 cells: A + ramp FBP", "ms_projection": t_a,
           "ms_fbp": t_f, "value": work / ((t_a + t_f) / 1e3) / 1e9, "unit": UNIT}
    if cpu:
        from oracle import refcpu
        if refcpu.available():
            opts = P.options.cpu().numpy()
            t0 = time.perf_counter()
            s = refcpu.dd2d("A", img[None, None], opts, ang_np)
            t1 = time.perf_counter()
            sf = _cpu_filter_rows(s.astype(np.float32), P.weight.cpu().numpy(), P.filter.cpu().numpy())
            refcpu.dd2d("BW", sf.astype(np.float32), opts, ang_np)
            t2 = time.perf_counter()
            out["reference_cpu"] = {"ms_projection": (t1 - t0) * 1e3, "ms_fbp": (t2 - t1) * 1e3,
                                    "value": work / (t2 - t0) / 1e9, "cores": os.cpu_count() or 1,
                                    "sample": "the full workload (the reference's CPU operators, torch conv2d filter)"}
    return out


def config_c2(dev, cpu: bool):
    """3D cone-flat FDK: 256x256x64 (1 mm) 3D Shepp-Logan + 20 seeded
    ellipsoids, 720 views, flat detector 384x96 of 1.5 mm, SOD 500, SDD 1000:
    projection, then FDK (cosine weight, ramp filter, weighted
    backprojection).  value = 256^2 * 64 * 720 / (t_A + t_FDK)."""
    import numpy as np
    import torch
    from xrecon_b200 import geometry as G
    from xrecon_b200.phantom import shepp_logan_plus_ellipsoids3d
    from xrecon_b200.projector import Projector3d
    P = Projector3d(G.Volume3d((256, 256, 64), 1.0),
                    G.ConeBeam3d(G.Detector3d((384, 96), (1.5, 1.5)), 500.0, 1000.0, "flat")).to(dev)
    vol = shepp_logan_plus_ellipsoids3d((64, 256, 256), 20, seed=2).astype(np.float32)
    ang_np = (np.arange(720) * (2 * np.pi / 720)).astype(np.float32)
    x = torch.from_numpy(vol)[None, None].to(dev)
    a = torch.from_numpy(ang_np).to(dev)
    sino = P.projection(x, a)
    t_a = _timed_ms(lambda: P.projection(x, a), 5)
    t_f = _timed_ms(lambda: P.filtered_backprojection(sino, a), 5)
    work = 256 * 256 * 64 * 720
    out = {"workload": "3D cone-flat 256x256x64, 720 views, 384x96 det: A + FDK", "ms_projection": t_a,
           "ms_fdk": t_f, "value": work / ((t_a + t_f) / 1e3) / 1e9, "unit": UNIT}
    del sino
    if cpu:
        from oracle import refcpu
        if refcpu.available():
            nv = 8
            sub = ang_np[:: 720 // nv][:nv].copy()
            opts = P.options.cpu().numpy()
            t0 = time.perf_counter()
            s = refcpu.dd3d("A", vol[None, None], opts, sub)
            t1 = time.perf_counter()
            sf = _cpu_filter_rows(s.astype(np.float32), P.weight.cpu().numpy(), P.filter.cpu().numpy())
            refcpu.dd3d("BW", sf.astype(np.float32), opts, sub)
            t2 = time.perf_counter()
            k = 720 / nv
            out["reference_cpu"] = {"ms_projection": (t1 - t0) * k * 1e3, "ms_fdk": (t2 - t1) * k * 1e3,
                                    "value": work / ((t2 - t0) * k) / 1e9, "cores": os.cpu_count() or 1,
                                    "sample": f"{nv} of 720 views, scaled by the view count"}
    return out


def config_c3(dev, cpu: bool, steps: int = 50):
    """Differentiable 3D cone-arc least squares: B=8 volumes of 128x128x32
    (1 mm) of seeded ellipsoids, 360 views, arc detector 256x64 of 1.5 mm, SOD
    500, SDD 1000; data = projection + Poisson noise at 1e5 photons.  One
    gradient step of ||Ax - y||^2 / 2 + 1e-3 TV(x) through the view-chunked
    Function (A in the forward, A again and A^T in the backward), and the
    50-step loop.  value = 8 * 128^2 * 32 * 360 / (t_A + t_AT)."""
    import numpy as np
    import torch
    from xrecon_b200 import backend as BK
    from xrecon_b200 import geometry as G
    from xrecon_b200.functions import projection_least_squares
    from xrecon_b200.phantom import ellipsoid_volume_torch, random_ellipsoids3d
    det = G.Detector3d((256, 64), (1.5, 1.5))
    opts = torch.tensor(G.pack_options3d(G.Volume3d((128, 128, 32), 1.0), G.ConeBeam3d(det, 500.0, 1000.0, "arc")),
                        dtype=torch.float32, device=dev)
    ang = (torch.arange(360, device=dev, dtype=torch.float64) * (2 * np.pi / 360)).float()
    xs = [ellipsoid_volume_torch((32, 128, 128), random_ellipsoids3d(8, seed=100 + i, density=(0.0, 1.0)), dev)
          for i in range(8)]
    x_true = (torch.stack(xs)[:, None] * 0.02).contiguous()
    g = torch.Generator(device=dev).manual_seed(5)
    p = BK.forward_projection3d(x_true, opts, ang)
    counts = torch.poisson(1e5 * torch.exp(-p), generator=g).clamp_min(1.0)
    y = -torch.log(counts / 1e5)
    t_a = _timed_ms(lambda: BK.forward_projection3d(x_true, opts, ang), 3)
    t_at = _timed_ms(lambda: BK.projection_transpose3d(p, opts, ang), 3)

    def tv(v, eps=1e-6):
        dz = v[:, :, 1:, :-1, :-1] - v[:, :, :-1, :-1, :-1]
        dy = v[:, :, :-1, 1:, :-1] - v[:, :, :-1, :-1, :-1]
        dx = v[:, :, :-1, :-1, 1:] - v[:, :, :-1, :-1, :-1]
        return torch.sqrt(dx * dx + dy * dy + dz * dz + eps).sum()

    # step size 1 / ||A^T A|| by power iteration
    v = torch.rand(x_true.shape, device=dev, generator=g)
    for _ in range(6):
        v = BK.projection_transpose3d(BK.forward_projection3d(v, opts, ang), opts, ang)
        lam = float(v.norm())
        v = v / lam
    step = 1.0 / lam
    x = torch.zeros_like(x_true, requires_grad=True)
    losses = []

    def loop(n):
        for _ in range(n):
            loss = projection_least_squares(x, y, opts, ang, view_chunk=24) + 1e-3 * tv(x)
            (gr,) = torch.autograd.grad(loss, x)
            with torch.no_grad():
                x.sub_(step * gr)
            losses.append(loss.detach())

    loop(1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    loop(steps)
    e1.record()
    torch.cuda.synchronize()
    t_loop = e0.elapsed_time(e1)
    work = 8 * 128 * 128 * 32 * 360
    out = {"workload": "3D cone-arc B=8 x 128x128x32, 360 views, 256x64 arc det: A + A^T gradient step",
           "ms_projection": t_a, "ms_projection_t": t_at, "value": work / ((t_a + t_at) / 1e3) / 1e9, "unit": UNIT,
           "ms_50_step_loop": t_loop * steps / 50.0 if steps != 50 else t_loop,
           "ms_per_gradient_step": t_loop / steps,
           "loss_first_last": [float(losses[0]), float(losses[-1])]}
    del p, counts, y, x
    if cpu:
        from oracle import refcpu
        if refcpu.available():
            nv = 4
            sub = ang.cpu().numpy()[:: 360 // nv][:nv].copy()
            o = opts.cpu().numpy()
            xt = x_true.cpu().numpy()
            t0 = time.perf_counter()
            s = refcpu.dd3d("A", xt, o, sub)
            t1 = time.perf_counter()
            refcpu.dd3d("AT", s.astype(np.float32), o, sub)
            t2 = time.perf_counter()
            k = 360 / nv
            out["reference_cpu"] = {"ms_projection": (t1 - t0) * k * 1e3, "ms_projection_t": (t2 - t1) * k * 1e3,
                                    "value": work / ((t2 - t0) * k) / 1e9, "cores": os.cpu_count() or 1,
                                    "sample": f"{nv} of 360 views of the B=8 batch, scaled by the view count"}
    return out


def baseline_configs(dev, cpu: bool):
    """The named configurations besides the headline one (which is the main
    line), each timed on this GPU and, with cpu, the reference's own CPU
    operators on a bounded sample of the same workload on this host."""
    out = {}
    for name, fn in (("c1_fan_flat_2d_fbp", config_c1), ("c2_cone_flat_fdk", config_c2),
                     ("c3_cone_arc_least_squares", config_c3)):
        try:
            out[name] = fn(dev, cpu)
        except Exception as exc:  # a side measurement must not cost the main line
            out[name] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    return out


def run_sharded_arm(args, rank: int, world: int, local_rank: int):
    """Strong scaling of the headline workload: one problem split over the
    ranks.  Each rank projects its share of the views, the view shards are
    all-gathered over NCCL (one collective), and each rank backprojects its
    z-slab of the volume with the full sinogram.  value = the whole
    problem's voxel-views / the slowest rank's step time."""
    import torch
    import torch.distributed as dist
    from xrecon_b200 import backend as BK
    from xrecon_b200 import distributed as XD
    from xrecon_b200.phantom import ellipsoid_volume_torch, random_ellipsoids3d
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    P = make_projector().to(dev)
    opts = P.options
    vol = ellipsoid_volume_torch((WL["D"], WL["H"], WL["W"]), random_ellipsoids3d(20, seed=0, density=(0.0, 1.0)),
                                 dev)[None, None].contiguous()
    ang = torch.from_numpy(angles_np(args.views, args.contiguous_views)).to(dev)
    nv = ang.numel()
    stream = torch.cuda.current_stream(dev)
    events = []

    def mark(_name):
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        events[-1].append(e)

    def step():
        events.append([torch.cuda.Event(enable_timing=True)])
        events[-1][0].record(stream)
        return XD.sharded_projection_backprojection(BK.forward_projection3d, BK.backward_projection3d, vol, opts, ang,
                                                    rank, world, marks=mark)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    events.clear()
    clocks = ClockSampler(local_rank)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    clk = clocks.stop()
    dist.barrier()
    t_step = sum(e[0].elapsed_time(e[3]) for e in events) / args.steps / 1e3
    phases = [sum(e[i].elapsed_time(e[i + 1]) for e in events) / args.steps for i in range(3)]
    t_step = XD.max_over_ranks(t_step, dev)
    phases = [XD.max_over_ranks(p, dev) for p in phases]
    value = nvox() * nv / t_step / 1e9
    hbm, src = peaks()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random ellipsoids)",
            "config": {"workload": WORKLOAD_NAME, "views": nv, "parallelism": f"views x{world} for A, "
                       f"NCCL all_gather of the sinogram, z-slabs x{world} for B",
                       "ms_projection_max_rank": phases[0], "ms_all_gather_max_rank": phases[1],
                       "ms_backprojection_max_rank": phases[2],
                       "l2": "inputs larger than L2 (volume 256 MiB, sinogram 1.41 GiB)"},
            "roofline": {"bound": "hbm", "peak": hbm, "unit": "GB/s", "peak_source": src,
                         "achieved": 2 * algo_bytes_op(dict(WL, V=nv)) / t_step / 1e9 / world,
                         "frac": 2 * algo_bytes_op(dict(WL, V=nv)) / t_step / 1e9 / world / hbm, "traffic": None,
                         "note": "per GPU: the step's algorithmic bytes / world / step time"},
            "e2e": None, "gpu_launches": None, "clocks": clk,
        }
        print(json.dumps(line))
    return 0


def run_gpu_arm(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch
    import torch.distributed as dist
    from xrecon_b200.phantom import ellipsoid_volume_torch, random_ellipsoids3d

    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    P = make_projector().to(dev)
    D, H, W = WL["D"], WL["H"], WL["W"]
    vol = ellipsoid_volume_torch((D, H, W), random_ellipsoids3d(20, seed=rank, density=(0.0, 1.0)), dev)
    vol = vol[None, None].contiguous()
    ang = torch.from_numpy(angles_np(args.views, args.contiguous_views)).to(dev)
    nv = ang.numel()

    def step(x):
        s = P.projection(x, ang)
        return P.backprojection(s, ang)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        step(vol)
    torch.cuda.synchronize()

    # timed region: per-operator CUDA events on the launching stream
    stream = torch.cuda.current_stream(dev)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    from xrecon_b200 import _native
    launches0 = _native.launch_count()
    e0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        s = P.projection(vol, ang)
        ev[i][1].record(stream)
        r = P.backprojection(s, ang)
        ev[i][2].record(stream)
        del s, r
    e1.record(stream)
    launches = _native.launch_count() - launches0
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    t_total = e0.elapsed_time(e1) / 1e3
    t_a = sum(e[0].elapsed_time(e[1]) for e in ev) / args.steps / 1e3
    t_b = sum(e[1].elapsed_time(e[2]) for e in ev) / args.steps / 1e3
    t_step = t_total / args.steps
    if world > 1:
        t = torch.tensor([t_step], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_step = float(t.item())
    value = world * nvox() * nv / t_step / 1e9

    # End-to-end through the public API with host buffers: every step copies
    # its volume in from pinned host memory and its result back.  The copies
    # run on their own streams, double-buffered, so that step i + 1's input
    # and step i's result cross PCIe while the GPU computes (the way a
    # pipeline feeding volumes would run); the timed region spans all the
    # steps' copies, the first input's and the last result's included.
    e2e_value = None
    if not args.no_e2e:
        host_vol = [vol.cpu().pin_memory() for _ in range(2)]
        host_out = [torch.empty_like(host_vol[0]).pin_memory() for _ in range(2)]
        dvol = [torch.empty_like(vol) for _ in range(2)]
        h2d_s, d2h_s = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        h2d_done = [torch.cuda.Event() for _ in range(2)]
        a_done = [torch.cuda.Event() for _ in range(2)]
        out_ready = [torch.cuda.Event() for _ in range(2)]
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps = args.steps

        def h2d(i):
            j = i % 2
            with torch.cuda.stream(h2d_s):
                if i >= 2:
                    h2d_s.wait_event(a_done[j])  # step i - 2's projection has read dvol[j]
                dvol[j].copy_(host_vol[j], non_blocking=True)
                h2d_done[j].record(h2d_s)

        barrier()
        torch.cuda.synchronize()
        f0.record(stream)
        h2d_s.wait_stream(stream)
        d2h_s.wait_stream(stream)
        h2d(0)
        for i in range(e2e_steps):
            j = i % 2
            if i + 1 < e2e_steps:
                h2d(i + 1)
            stream.wait_event(h2d_done[j])
            sino = P.projection(dvol[j], ang)
            a_done[j].record(stream)
            out = P.backprojection(sino, ang)
            out_ready[j].record(stream)
            with torch.cuda.stream(d2h_s):
                d2h_s.wait_event(out_ready[j])
                host_out[j].copy_(out, non_blocking=True)
                out.record_stream(d2h_s)
            del sino, out
        stream.wait_stream(h2d_s)
        stream.wait_stream(d2h_s)
        f1.record(stream)
        torch.cuda.synchronize()
        t_e2e = f0.elapsed_time(f1) / 1e3 / e2e_steps
        if world > 1:
            t = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e_value = world * nvox() * nv / t_e2e / 1e9
    vol_bytes = vol.numel() * 4

    # Half-precision storage forms of the same step, FP32 accumulation,
    # reported beside the FP32 number:
    #   bf16: volume, sinogram and backprojected volume in BF16;
    #   fp16: volume and sinogram in FP16, the backprojected volume in FP32
    #         (the unscaled sum over 1440 views exceeds FP16's range).
    half = {}
    if not args.no_bf16:
        from xrecon_b200 import _native as NT

        def step_fp16(x):
            s16 = P.projection(x, ang)
            return NT.apply(3, "B", s16, P._host().struct, ang, out_dtype=torch.float32)

        ref32 = step(vol)
        for name, dt, fn, vout in (("bf16", torch.bfloat16, step, "bf16"),
                                   ("fp16", torch.float16, step_fp16, "fp32")):
            try:
                vol16 = vol.to(dt)
                fn(vol16)
                torch.cuda.synchronize()
                g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                nb = max(1, min(args.steps, 3))
                g0.record(stream)
                for _ in range(nb):
                    out16 = fn(vol16)
                g1.record(stream)
                torch.cuda.synchronize()
                t16 = g0.elapsed_time(g1) / 1e3 / nb
                rel = float((out16.float() - ref32).norm() / ref32.norm())
                half[name] = {"value": world * nvox() * nv / t16 / 1e9, "unit": UNIT, "ms_per_step": t16 * 1e3,
                              "rel_l2_vs_fp32": rel, "backprojected_volume": vout}
                del vol16, out16
            except Exception as exc:  # a storage form must not cost the main line
                half[name] = {"error": f"{type(exc).__name__}: {exc}"[:200]}
        del ref32

    hbm, src = peaks()
    dom_t = max(t_a, t_b)
    dom = "cell_tma3d_kernel (projection A)" if t_a >= t_b else "vox_prefix3d_kernel (backprojection B)"
    # what holds the kernel below the HBM roofline, from its ncu profile
    # (profiles/cell_tma3d_A_cone_flat_64views.md, vox_prefix3d_B_cone_flat_64views.md)
    limiter = ("instruction issue: ~70 % issue active, 'not selected' stalls, DRAM ~3 % of peak"
               if t_a >= t_b else
               "table-lookup latency and issue: ~67 % issue active, long-scoreboard (L1 hit) stalls, DRAM idle")
    wl = dict(WL, V=nv)
    achieved = algo_bytes_op(wl) / dom_t / 1e9
    traffic = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        tj = json.loads(tp.read_text())
        full = tj.get("A" if t_a >= t_b else "B")
        # recorded at the full view count; scaled for a profiling subset
        traffic = None if full is None else full * nv / tj.get("views", WL["V"])

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random ellipsoids)",
        "config": {"workload": WORKLOAD_NAME if nv == WL["V"] else f"{WORKLOAD_NAME} (profiling subset: {nv} views)",
                   "volume": [WL["D"], WL["H"], WL["W"]], "views": nv,
                   "detector": [WL["Nv"], WL["Nu"]], "ms_projection": t_a * 1e3,
                   "ms_backprojection": t_b * 1e3,
                   "l2": "inputs larger than L2 (volume 256 MiB, sinogram 1.41 GiB)",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "limiter": limiter, "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": algo_bytes_op(wl),
                     # every voxel and detector cell touched once per operator
                     "compulsory_bytes_per_launch": (nvox(wl) + wl["V"] * wl["Nu"] * wl["Nv"]) * 4},
        "e2e": None if e2e_value is None else {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": vol_bytes,
                                               "d2h_bytes_per_step": vol_bytes},
        "gpu_launches": launches,
        "clocks": clk,
    }
    line.update(half)
    if not args.no_ops:
        line["operators"] = operator_times(P, vol, ang, nv)
    if not args.no_ragged and world == 1:
        line["ragged_fan_arc_batch"] = ragged_measure(dev)
    if not args.no_sysmat and world == 1:
        line["system_matrix_2d_fan_flat"] = sysmat_measure(dev)
    if not args.no_rebin and world == 1:
        line["rebin_fan_to_parallel"] = rebin_measure(P, vol, ang)
    if not args.no_helical and world == 1:
        line["helical_arc_512x512x128_736x64_5x1152views"] = helical_measure(dev)
    if not args.no_configs and world == 1:
        line["configs"] = baseline_configs(dev, cpu=(rank == 0 and not args.no_cpu))
    if rank == 0 and world == 1 and not args.no_cpu:
        sample = cpu_reference_sample(4, vol.cpu().numpy())
        line["cpu_baseline"] = {k: v for k, v in sample.items() if k != "seconds"} if sample else None
    if rank == 0:
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-bf16", action="store_true", help="skip the BF16/FP16-storage measurements")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    ap.add_argument("--no-ragged", action="store_true", help="skip the ragged 2D batch measurement")
    ap.add_argument("--no-ops", action="store_true", help="skip the per-operator timings")
    ap.add_argument("--no-sysmat", action="store_true", help="skip the system-matrix export timing")
    ap.add_argument("--no-rebin", action="store_true", help="skip the rebinning timing")
    ap.add_argument("--no-helical", action="store_true", help="skip the helical projector timings")
    ap.add_argument("--helical-only", action="store_true",
                    help="profiling: only the helical projector timings (one JSON line)")
    ap.add_argument("--helical-turns", type=int, default=None,
                    help="profiling: turns of the helical scan (default 5) with --helical-only")
    ap.add_argument("--views", type=int, default=None,
                    help="profiling: an evenly strided subset of the workload's views")
    ap.add_argument("--contiguous-views", action="store_true",
                    help="profiling: with --views, the first neighbouring views instead of a strided subset")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other named configurations (2D FBP, 3D FDK, cone-arc least squares)")
    ap.add_argument("--only", choices=["c1", "c2", "c3"], default=None,
                    help="profiling: only one of the other named configurations (one JSON line)")
    ap.add_argument("--plain", action="store_true",
                    help="profiling: run every operator through the plain (non-staged) kernels")
    ap.add_argument("--replicas", action="store_true",
                    help="with several GPUs: independent replicas of the workload (weak scaling) instead of one "
                         "problem split over the GPUs (strong scaling, the default)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    if args.plain:
        from xrecon_b200 import _native
        _native.set_plain_kernels(True)
    if args.only:
        import torch
        fn = {"c1": config_c1, "c2": config_c2, "c3": config_c3}[args.only]
        print(json.dumps({args.only: fn(torch.device("cuda:0"), not args.no_cpu)}))
        return 0
    if args.helical_only:
        import torch
        print(json.dumps({"helical_arc_512x512x128_736x64_5x1152views":
                          helical_measure(torch.device("cuda:0"), turns=args.helical_turns)}))
        return 0
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if world > 1 and not args.replicas:
            return run_sharded_arm(args, rank, world, local_rank)
        return run_gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
