"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run where the XRecon reference tree is importable, naming its root in
XRECON_REFERENCE_ROOT:

    XRECON_REFERENCE_ROOT=<reference tree> python tests/golden/make_golden.py

The reference's own Python package (xrecon/projector/*.py, pure Python) is
imported from the reference tree with its native module ``xrecon_C`` served
by the reference's own C++ CPU kernels (src/cpu/*.cpp compiled by
oracle/build_oracle.py into oracle/_ref/).  So every number stored here comes
from the reference's code path on CPU:

* dd2d_<geom>.npz / dd3d_<geom>.npz: seeded inputs and the outputs of the six
  operators (forward_projection, projection_transpose, backward_projection,
  weighted_backward_projection and the two backprojection transposes);
* fbp2d_<case>.npz / fdk3d_<case>.npz: Projector.filtered_backprojection
  results (TF32 is irrelevant: this is the CPU conv path);
* options.npz: the packed options vectors of Projector2d/3d for the benchmark
  geometries; filters.npz: the filter tables;
* sysmat{2,3}d_<geom>.npz: the reference's sparse projection matrices
  (system_matrix2d_cpu / system_matrix3d_cpu) for small shifted geometries
  (``python tests/golden/make_golden.py sysmat`` writes only these);
* rebin_<case>.npz: the reference's fan/helical -> parallel rebinning
  (xrecon/utils/rebin.py, pure torch) on seeded inputs
  (``python tests/golden/make_golden.py rebin``);
* helical_host.npz: HelicalProjector3d's packed options, weight, filter and
  source positions (``python tests/golden/make_golden.py helical_host``);
* filters_sweep.npz: the reference's filter tables (filters.py:19-71) for
  odd and even detector counts and several spacings
  (``python tests/golden/make_golden.py filters``);
* autograd{2,3}d_<geom>.npz: gradients of the reference's twelve autograd
  Functions (xrecon/projector/functions.py:96-302) for a seeded input and
  upstream gradient (``python tests/golden/make_golden.py autograd``).
The reference's helical operators themselves are CUDA only; their outputs
are recorded on a GPU by tests/golden/make_golden_helical.py.
"""
from __future__ import annotations

import math
import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
if not os.environ.get("XRECON_REFERENCE_ROOT"):
    sys.exit("set XRECON_REFERENCE_ROOT to the XRecon reference tree")
REF_ROOT = Path(os.environ["XRECON_REFERENCE_ROOT"])
sys.path.insert(0, str(ROOT))

from oracle import refcpu  # noqa: E402


def import_reference():
    """Import the reference package with xrecon_C served by its CPU kernels."""
    sys.modules["xrecon_C"] = refcpu.RefXreconC()
    sys.path.insert(0, str(REF_ROOT))
    import xrecon.projector.filters as rfilters  # noqa: F401
    from xrecon.projector.projector import Projector2d
    from xrecon.projector.projector3d import Projector3d
    import xrecon.projector.geometry as rgeom
    return Projector2d, Projector3d, rgeom, rfilters


OPS2D = {"A": "projection", "AT": "projection_t", "B": "backprojection", "BW": "backprojection_weighted",
         "BT": "backprojection_t", "BWT": "backprojection_weighted_t"}


def angles_set(V: int, offset: float = 0.1) -> np.ndarray:
    a = (np.arange(V) * (2 * np.pi / V) + offset).astype(np.float32)
    special = np.array([0.0, np.pi / 4, np.pi / 2, 3 * np.pi / 4, np.pi, 5 * np.pi / 4], np.float32)
    return np.concatenate([a, special]).astype(np.float32)


def main():
    P2, P3, G, F = import_reference()
    rng = np.random.default_rng(20261203)

    # ---------------------------------------------------------------- 2D ops
    for scan in ("parallel", "flat", "arc"):
        if scan == "parallel":
            geo = G.ParallelBeam2d(G.Detector2d(53, 1.7, 0.25))
        else:
            geo = G.FanBeam2d(G.Detector2d(53, 1.7, 0.25), 500.0, 1000.0, scan)
        P = P2(G.Volume2d((37, 29), (1.0, 1.1), (0.3, -0.2)), geo)
        ang = angles_set(18)
        img = rng.random((2, 1, 29, 37)).astype(np.float32)
        sino = rng.random((2, 1, ang.size, 53)).astype(np.float32)
        at = torch.from_numpy(ang)
        out = {"options": P.options.numpy(), "angles": ang, "image": img, "sino": sino}
        for op, meth in OPS2D.items():
            x = img if op in ("A", "BT", "BWT") else sino
            out[op] = getattr(P, meth)(torch.from_numpy(x), at).numpy()
        np.savez_compressed(HERE / f"dd2d_{scan}.npz", **out)

    # ---------------------------------------------------------------- 3D ops
    for scan in ("parallel", "flat", "arc"):
        det = G.Detector3d((41, 13), (1.5, 1.3), (0.25, -0.5))
        geo = G.ParallelBeam3d(det) if scan == "parallel" else G.ConeBeam3d(det, 500.0, 1000.0, scan)
        P = P3(G.Volume3d((23, 19, 11), (1.0, 1.1, 0.9), (0.2, -0.3, 0.5)), geo)
        ang = angles_set(10)
        img = rng.random((1, 1, 11, 19, 23)).astype(np.float32)
        sino = rng.random((1, 1, ang.size, 13, 41)).astype(np.float32)
        at = torch.from_numpy(ang)
        out = {"options": P.options.numpy(), "angles": ang, "image": img, "sino": sino}
        for op, meth in OPS2D.items():
            x = img if op in ("A", "BT", "BWT") else sino
            out[op] = getattr(P, meth)(torch.from_numpy(x), at).numpy()
        np.savez_compressed(HERE / f"dd3d_{scan}.npz", **out)

    # ------------------------------------------------------------- FBP / FDK
    from xrecon.utils.phantom import phantom as rphantom  # pure numpy
    img = torch.from_numpy(rphantom(64, dim=2)).float()[None, None]
    cases2d = [("flat_ramp", "flat", "ramp", 90, 2 * np.pi, False),
               ("arc_ramp", "arc", "ramp", 90, 2 * np.pi, False),
               ("parallel_shepplogan", "parallel", "shepplogan", 60, np.pi, False),
               ("flat_hann", "flat", "hann", 90, 2 * np.pi, False),
               ("flat_parker", "flat", "ramp", 80, np.pi + 0.6, True)]
    for name, scan, filt, V, rng_ang, parker in cases2d:
        if scan == "parallel":
            geo = G.ParallelBeam2d(G.Detector2d(96, 1.0))
        else:
            geo = G.FanBeam2d(G.Detector2d(96, 2.0), 500.0, 1000.0, scan)
        P = P2(G.Volume2d(64, 1.0), geo, filter_type=filt)
        ang = torch.from_numpy((np.arange(V) * (rng_ang / V)).astype(np.float32))
        sino = P.projection(img, ang)
        recon = P.filtered_backprojection(sino, ang, parker=parker)
        np.savez_compressed(HERE / f"fbp2d_{name}.npz", options=P.options.numpy(), angles=ang.numpy(),
                            sino=sino.numpy(), weight=P.weight.numpy(), filter=P.filter.numpy(),
                            parker=P.parker_weight(ang).numpy() if parker else np.zeros(0, np.float32),
                            recon=recon.numpy())

    vol = torch.from_numpy(np.ascontiguousarray(
        np.transpose(rphantom((32, 32, 8), dim=3), (2, 0, 1)))).float()[None, None]
    for name, scan in (("flat", "flat"), ("arc", "arc")):
        geo = G.ConeBeam3d(G.Detector3d((48, 12), (1.5, 1.5)), 500.0, 1000.0, scan)
        P = P3(G.Volume3d((32, 32, 8), 1.0), geo)
        ang = torch.from_numpy((np.arange(60) * (2 * np.pi / 60)).astype(np.float32))
        sino = P.projection(vol, ang)
        recon = P.filtered_backprojection(sino, ang)
        np.savez_compressed(HERE / f"fdk3d_{name}.npz", options=P.options.numpy(), angles=ang.numpy(),
                            sino=sino.numpy(), weight=P.weight.numpy(), filter=P.filter.numpy(),
                            recon=recon.numpy())

    # ------------------------------------------------- packing + filter tables
    opts = {}
    opts["c1_2d_flat"] = P2(G.Volume2d(256, 1.0), G.FanBeam2d(G.Detector2d(256, 2.0), 500., 1000., "flat")).options.numpy()
    opts["c2_3d_flat"] = P3(G.Volume3d((256, 256, 64), 1.0),
                            G.ConeBeam3d(G.Detector3d((384, 96), 1.5), 500., 1000., "flat")).options.numpy()
    opts["c3_3d_arc"] = P3(G.Volume3d((128, 128, 32), 1.0),
                           G.ConeBeam3d(G.Detector3d((256, 64), 1.5), 500., 1000., "arc")).options.numpy()
    opts["c4_2d_arc"] = P2(G.Volume2d(384, 512 / 384), G.FanBeam2d(G.Detector2d(500, 1.3, 0.5), 450., 900., "arc")).options.numpy()
    opts["c5_3d_flat"] = P3(G.Volume3d((512, 512, 256), 0.75),
                            G.ConeBeam3d(G.Detector3d((1024, 256), 0.8), 595., 1085., "flat")).options.numpy()
    opts["x_3d_parallel"] = P3(G.Volume3d((40, 30, 20), (1.0, 1.2, 0.8), (0.5, -1, 2)),
                               G.ParallelBeam3d(G.Detector3d((64, 24), (1.1, 0.9), (0.3, -0.7)))).options.numpy()
    opts["x_2d_parallel"] = P2(G.Volume2d((40, 30), (1.0, 1.2), (0.5, -1)),
                               G.ParallelBeam2d(G.Detector2d(64, 1.1, 0.3))).options.numpy()
    opts["x_3d_arc_shift"] = P3(G.Volume3d((40, 30, 20), (1.0, 1.2, 0.8), (0.5, -1, 2)),
                                G.ConeBeam3d(G.Detector3d((64, 24), (1.1, 0.9), (0.3, -0.7)), 600., 1100., "arc")).options.numpy()
    np.savez_compressed(HERE / "options.npz", **opts)

    filt = {}
    for name in ("ramp", "shepplogan", "cosine", "hamming", "hann"):
        filt[name] = F.filter_generate(96, 0.75, name, torch.float32).numpy()
    np.savez_compressed(HERE / "filters.npz", **filt)
    print("fixtures written to", HERE)


def make_sysmat():
    """sysmat{2,3}d_<geom>.npz: the reference's system_matrix2d/3d triplets
    (its own CPU code through oracle/_ref) for small shifted geometries."""
    P2, P3, G, F = import_reference()
    ang = angles_set(10, 0.2)
    for scan in ("parallel", "flat", "arc"):
        if scan == "parallel":
            geo2 = G.ParallelBeam2d(G.Detector2d(32, 1.1, 0.4))
            geo3 = G.ParallelBeam3d(G.Detector3d((16, 6), (1.1, 0.9), (0.3, -0.4)))
        else:
            geo2 = G.FanBeam2d(G.Detector2d(32, 2.0, 0.4), 300.0, 600.0, scan)
            geo3 = G.ConeBeam3d(G.Detector3d((16, 6), (1.6, 1.4), (0.3, -0.4)), 300.0, 600.0, scan)
        for dim, P in ((2, P2(G.Volume2d((24, 20), (1.0, 1.1), (0.5, -0.5)), geo2)),
                       (3, P3(G.Volume3d((12, 10, 6), (1.0, 1.1, 1.2), (0.5, -0.5, 0.5)), geo3))):
            opts = P.options.numpy()
            r, c, v, shape = refcpu.system_matrix(dim, opts, ang)
            np.savez_compressed(HERE / f"sysmat{dim}d_{scan}.npz", options=opts, angles=ang, rows=r, cols=c,
                                vals=v, shape=np.array(shape, np.int64))
    print("system-matrix fixtures written to", HERE)


def make_rebin():
    """rebin_<case>.npz: the reference's fan_to_parallel_rebin /
    helical_fan_to_parallel_rebin (xrecon/utils/rebin.py, pure torch, run on
    the CPU) on seeded inputs."""
    sys.path.insert(0, str(REF_ROOT))
    import importlib.util
    spec = importlib.util.spec_from_file_location("xrecon_rebin_ref", REF_ROOT / "xrecon" / "utils" / "rebin.py")
    R = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(R)
    rng = np.random.default_rng(21)
    cases = {
        "arc4d": ("arc", (1, 1, 90, 64), 0.004, {}),
        "flat5d": ("flat", (2, 1, 72, 5, 48), 1.5, dict(output_det_count=40, output_det_shift=0.7)),
        "arc5d_grid": ("arc", (1, 2, 60, 3, 50), 0.004,
                       dict(output_angles=torch.linspace(0.3, 5.0, 33), output_det_spacing=3.0)),
    }
    for name, (det, shape, du, kw) in cases.items():
        V = shape[2]
        ang = torch.arange(V, dtype=torch.float32) * (2 * np.pi / V) + 0.1
        sino = torch.from_numpy(rng.random(shape).astype(np.float32))
        out, oa, t = R.fan_to_parallel_rebin(sino, ang, 500.0, du, 0.3 * du, det, **kw)
        extra = {k: (v.numpy() if torch.is_tensor(v) else np.array(v)) for k, v in kw.items()}
        np.savez_compressed(HERE / f"rebin_{name}.npz", sino=sino.numpy(), angles=ang.numpy(), iso_source=500.0,
                            det_spacing=du, det_shift=0.3 * du, detector_type=det, out=out.numpy(),
                            out_angles=oa.numpy(), t=t.numpy(), **{f"kw_{k}": v for k, v in extra.items()})
    V = 80
    ang = torch.arange(V, dtype=torch.float32) * (2 * np.pi / V)
    zsrc = torch.linspace(-20.0, 20.0, V)
    sino = torch.from_numpy(rng.random((1, 1, V, 4, 40)).astype(np.float32))
    oa_in = torch.linspace(-0.2, 6.5, 50)
    out, oa, t, z = R.helical_fan_to_parallel_rebin(sino, ang, zsrc, 550.0, 0.005, 0.0, "arc", output_angles=oa_in)
    np.savez_compressed(HERE / "rebin_helical.npz", sino=sino.numpy(), angles=ang.numpy(), source_z=zsrc.numpy(),
                        out_angles_in=oa_in.numpy(), out=out.numpy(), out_angles=oa.numpy(), t=t.numpy(),
                        out_source_z=z.numpy())
    print("rebinning fixtures written to", HERE)


HELICAL_HOST_CASES = {
    # name: (constructor keyword arguments, number of views)
    "one_turn": (dict(image_size=(32, 32, 16), num_det=(48, 8), pix_size=(2.0, 2.0, 1.0), det_size=(2.4, 2.0),
                      iso_source=300.0, source_detector=600.0, pixshift=(0.1, -0.2, 0.3), binshift=(0.3, -0.1),
                      pitch=8.0, z0=-8.0), 192),
    "auto_tang": (dict(image_size=(24, 20, 12), num_det=(40, 6), pix_size=(2.5, 2.5, 1.5), det_size=(3.0, 2.5),
                       iso_source=320.0, source_detector=640.0, pitch=12.0, z0=-9.0, helical_view_mode="auto",
                       helical_weight_mode="tang3d", helical_tang_k=3.0, helical_tang_blend=0.6,
                       filter_type="hann"), 150),
    "half_scan": (dict(image_size=(32, 32, 16), num_det=(48, 8), pix_size=(2.0, 2.0, 1.0), det_size=(2.4, 2.0),
                       iso_source=300.0, source_detector=600.0, pitch=14.0, z0=-10.0, helical_view_mode="half",
                       helical_halfscan_coef=1.1, filter_type="shepplogan"), 180),
}


def make_helical_host():
    """helical_host.npz: the reference HelicalProjector3d's packed options,
    cell weight, filter, source_position and mean angle step
    (xrecon/projector/projector3d.py:289-576, pure Python) for a few
    configurations; no operator is run."""
    sys.modules["xrecon_C"] = refcpu.RefXreconC()
    sys.path.insert(0, str(REF_ROOT))
    from xrecon.projector.projector3d import HelicalProjector3d
    out = {}
    for name, (kw, V) in HELICAL_HOST_CASES.items():
        P = HelicalProjector3d(**kw)
        ang = torch.arange(V, dtype=torch.float32) * (2 * np.pi / 96) + 0.05
        out[f"{name}_options"] = P.options.numpy()
        out[f"{name}_weight"] = P.weight.numpy()
        out[f"{name}_filter"] = P.filter.numpy()
        out[f"{name}_angles"] = ang.numpy()
        out[f"{name}_source_pos"] = P.source_position(ang).numpy()
        out[f"{name}_mean_step"] = np.float32(P._mean_angle_step(ang).item())
    np.savez_compressed(HERE / "helical_host.npz", **out)
    print("helical host fixtures written to", HERE)


FILTER_SWEEP = [(n, du) for n in (7, 64, 255, 1024) for du in (0.75, 2.3)]


def make_filters():
    """filters_sweep.npz: filter_generate(Nu, du, name) of the reference for
    FILTER_SWEEP x the five filter names, keyed "<name>_<Nu>_<du>"."""
    _, _, _, F = import_reference()
    out = {}
    for name in ("ramp", "shepplogan", "cosine", "hamming", "hann"):
        for n, du in FILTER_SWEEP:
            out[f"{name}_{n}_{du}"] = F.filter_generate(n, du, name, torch.float32).numpy()
    np.savez_compressed(HERE / "filters_sweep.npz", **out)
    print("filter sweep written to", HERE)


FUNCTIONS = {"A": "Projection", "AT": "ProjectionTranspose", "B": "BackProjection",
             "BW": "WeightedBackProjection", "BT": "BackProjectionTranspose",
             "BWT": "WeightedBackProjectionTranspose"}


def make_autograd():
    """autograd{2,3}d_<geom>.npz: for each of the reference's autograd
    Functions, a seeded input x, an upstream gradient u and
    d(sum(F(x) * u))/dx, taken by torch.autograd through the reference's own
    backward (its partner transpose binding, served here by its CPU
    kernels)."""
    P2, P3, G, _ = import_reference()
    import xrecon.projector.functions as RF
    rng = np.random.default_rng(20261204)
    for dim in (2, 3):
        for scan in ("parallel", "flat", "arc"):
            if dim == 2:
                det = G.Detector2d(31, 1.6, 0.3)
                geo = G.ParallelBeam2d(det) if scan == "parallel" else G.FanBeam2d(det, 450.0, 900.0, scan)
                P = P2(G.Volume2d((21, 17), (1.0, 1.2), (0.4, -0.3)), geo)
                img_shape, sino_of = (2, 1, 17, 21), (lambda V: (2, 1, V, 31))
            else:
                det = G.Detector3d((27, 9), (1.4, 1.2), (0.3, -0.4))
                geo = G.ParallelBeam3d(det) if scan == "parallel" else G.ConeBeam3d(det, 450.0, 900.0, scan)
                P = P3(G.Volume3d((15, 13, 7), (1.0, 1.1, 0.9), (0.2, 0.3, -0.4)), geo)
                img_shape, sino_of = (1, 1, 7, 13, 15), (lambda V: (1, 1, V, 9, 27))
            ang = angles_set(9, 0.2)
            at = torch.from_numpy(ang)
            out = {"options": P.options.numpy(), "angles": ang}
            for op, name in FUNCTIONS.items():
                in_shape, out_shape = ((img_shape, sino_of(ang.size)) if op in ("A", "BT", "BWT")
                                       else (sino_of(ang.size), img_shape))
                x = torch.from_numpy(rng.random(in_shape).astype(np.float32)).requires_grad_(True)
                u = torch.from_numpy(rng.random(out_shape).astype(np.float32))
                fn = getattr(RF, f"{name}{dim}d")
                y = fn.apply(x, P.options, at)
                (grad,) = torch.autograd.grad((y * u).sum(), x)
                out[f"{op}_x"] = x.detach().numpy()
                out[f"{op}_u"] = u.numpy()
                out[f"{op}_grad"] = grad.numpy()
            np.savez_compressed(HERE / f"autograd{dim}d_{scan}.npz", **out)
    print("autograd fixtures written to", HERE)


if __name__ == "__main__":
    if sys.argv[1:] == ["sysmat"]:
        make_sysmat()
    elif sys.argv[1:] == ["rebin"]:
        make_rebin()
    elif sys.argv[1:] == ["helical_host"]:
        make_helical_host()
    elif sys.argv[1:] == ["autograd"]:
        make_autograd()
    elif sys.argv[1:] == ["filters"]:
        make_filters()
    else:
        main()
        make_sysmat()
        make_rebin()
        make_helical_host()
