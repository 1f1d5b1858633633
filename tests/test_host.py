"""Host-side logic and the C ABI surface (CPU only, no kernel launches)."""
import ctypes
import re

import numpy as np
import pytest
import torch

from conftest import ROOT, load_golden
from xrecon_b200 import _native, filters, geometry as G
from xrecon_b200.projector import Projector2d, Projector3d, mean_angle_step, parker_weights


def _ref_geoms():
    return {
        "c1_2d_flat": (G.Volume2d(256, 1.0), G.FanBeam2d(G.Detector2d(256, 2.0), 500., 1000., "flat")),
        "c2_3d_flat": (G.Volume3d((256, 256, 64), 1.0), G.ConeBeam3d(G.Detector3d((384, 96), 1.5), 500., 1000., "flat")),
        "c3_3d_arc": (G.Volume3d((128, 128, 32), 1.0), G.ConeBeam3d(G.Detector3d((256, 64), 1.5), 500., 1000., "arc")),
        "c4_2d_arc": (G.Volume2d(384, 512 / 384), G.FanBeam2d(G.Detector2d(500, 1.3, 0.5), 450., 900., "arc")),
        "c5_3d_flat": (G.Volume3d((512, 512, 256), 0.75),
                       G.ConeBeam3d(G.Detector3d((1024, 256), 0.8), 595., 1085., "flat")),
        "x_3d_parallel": (G.Volume3d((40, 30, 20), (1.0, 1.2, 0.8), (0.5, -1, 2)),
                          G.ParallelBeam3d(G.Detector3d((64, 24), (1.1, 0.9), (0.3, -0.7)))),
        "x_2d_parallel": (G.Volume2d((40, 30), (1.0, 1.2), (0.5, -1)), G.ParallelBeam2d(G.Detector2d(64, 1.1, 0.3))),
        "x_3d_arc_shift": (G.Volume3d((40, 30, 20), (1.0, 1.2, 0.8), (0.5, -1, 2)),
                           G.ConeBeam3d(G.Detector3d((64, 24), (1.1, 0.9), (0.3, -0.7)), 600., 1100., "arc")),
    }


def test_packed_options_equal_reference():
    ref = load_golden("options")
    for name, (vol, geo) in _ref_geoms().items():
        P = (Projector2d if isinstance(vol, G.Volume2d) else Projector3d)(vol, geo)
        np.testing.assert_array_equal(P.options.numpy(), ref[name], err_msg=name)


def test_filter_tables_match_reference():
    ref = load_golden("filters")
    for name in ("ramp", "shepplogan", "cosine", "hamming", "hann"):
        got = filters.filter_generate(96, 0.75, name, torch.float32).numpy()
        np.testing.assert_allclose(got, ref[name], rtol=2e-6, atol=1e-7 * np.abs(ref[name]).max(), err_msg=name)


def test_filter_tables_match_reference_across_sizes():
    """Odd and even detector counts up to 1024 and two spacings: the windowed
    tables come from an FFT in FP64 on both sides, so they agree to the
    float32 rounding (1e-7 of the peak)."""
    ref = load_golden("filters_sweep")
    assert len(ref) == 40
    for key in sorted(ref):
        name, n, du = key.split("_")
        got = filters.filter_generate(int(n), float(du), name, torch.float32).numpy()
        assert got.shape == ref[key].shape, key
        np.testing.assert_allclose(got, ref[key], rtol=0, atol=3e-7 * np.abs(ref[key]).max(), err_msg=key)


def test_fbp_host_tables_match_reference():
    for case in ("flat_ramp", "arc_ramp", "parallel_shepplogan", "flat_hann"):
        g = load_golden(f"fbp2d_{case}")
        scan, filt = case.split("_")
        det = G.Detector2d(96, 2.0 if scan != "parallel" else 1.0)
        geo = G.ParallelBeam2d(det) if scan == "parallel" else G.FanBeam2d(det, 500.0, 1000.0, scan)
        P = Projector2d(G.Volume2d(64, 1.0), geo, filter_type=filt)
        np.testing.assert_array_equal(P.options.numpy(), g["options"])
        np.testing.assert_allclose(P.weight.numpy(), g["weight"], rtol=1e-6)
        np.testing.assert_allclose(P.filter.numpy(), g["filter"], rtol=2e-6, atol=1e-7 * np.abs(g["filter"]).max())
    g = load_golden("fbp2d_flat_parker")
    P = Projector2d(G.Volume2d(64, 1.0), G.FanBeam2d(G.Detector2d(96, 2.0), 500.0, 1000.0, "flat"))
    ang = torch.from_numpy(g["angles"])
    np.testing.assert_allclose(P.parker_weight(ang).numpy(), g["parker"], rtol=1e-6, atol=1e-7)


def test_mean_angle_step_wraps():
    a = torch.tensor([6.0, 6.2, 0.1, 0.3], dtype=torch.float64)
    step = mean_angle_step(a).item()
    assert abs(step - np.mean([0.2, 0.1 + 2 * np.pi - 6.2, 0.2])) < 1e-12


def test_parker_full_scan_is_ones():
    ang = torch.linspace(0, 2 * np.pi, 361, dtype=torch.float32)  # closed 2*pi scan
    w = parker_weights(ang, torch.linspace(-0.2, 0.2, 16), 16)
    assert torch.all(w == 1)
    with pytest.raises(ValueError):
        parker_weights(ang[:100], torch.linspace(-0.2, 0.2, 16), 16)


@pytest.mark.parametrize("gamma_max,overscan", [(0.1, 0.0), (0.3, 0.0), (0.3, 0.2), (0.45, 0.05)])
def test_parker_weights_sum_to_one_on_conjugate_rays(gamma_max, overscan):
    """The defining property of the short-scan weights (projector.py:208-246,
    Parker's sin^2 ramps with the overscan generalisation): a ray (beta,
    gamma) and its conjugate (beta + pi + 2 gamma, -gamma), both inside the
    scan, carry weights that add up to one.  FP64, seeded random rays."""
    rng = np.random.default_rng(17)
    R = np.pi + 2 * gamma_max + 2 * overscan
    for _ in range(200):
        g = rng.uniform(-gamma_max, gamma_max)
        b = rng.uniform(0, R - np.pi - 2 * g)  # so that the conjugate lies inside the scan too
        b2 = b + np.pi + 2 * g
        # the scan runs from 0 to R; the two extra columns fix gamma_max
        ang = torch.tensor([0.0, b, b2, R], dtype=torch.float64)
        gam = torch.tensor([g, -g, gamma_max, -gamma_max], dtype=torch.float64)
        w = parker_weights(ang, gam, 4)
        assert abs(float(w[1, 0] + w[2, 1]) - 1.0) < 1e-12, (b, g)


def _header_functions():
    text = (ROOT / "include" / "xrecon_b200.h").read_text()
    body = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xr_[a-z0-9_]+)\s*\(", body)))


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = _header_functions()
    assert "xr_dd3d" in names and "xr_dd2d" in names
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/xrecon_b200.h but not exported"
    assert _native.version().startswith("xrecon_b200")


def test_workspace_sizes_and_validation_without_gpu():
    lib = _native.lib()
    vals = load_golden("options")["c5_3d_flat"]
    g = _native.geom3d_from_values(vals)
    nb_a = lib.xr_dd3d_workspace_size(0, ctypes.byref(g), 1, 1440)
    nb_at = lib.xr_dd3d_workspace_size(1, ctypes.byref(g), 1, 1440)
    # forward needs the flipped image copy (FP32 for every storage type, since
    # half-precision images are widened once) plus the widened copy itself;
    # cone A^T the scaled sinogram
    assert nb_a > 2 * 512 * 512 * 256 * 4
    assert nb_at > 1440 * 256 * 1024 * 4
    bad = _native.geom3d_from_values(vals)
    bad.dx = -1.0
    rc = lib.xr_dd3d(0, ctypes.byref(bad), None, 0, None, 0, None, 1, 1, None, 0, None)
    assert rc == 1
    assert b"spacings" in lib.xr_last_error()
    near = _native.geom3d_from_values(vals)
    near.sod = 100.0  # source inside the image
    rc = lib.xr_dd3d(0, ctypes.byref(near), ctypes.c_void_p(1), 0, ctypes.c_void_p(1), 0, ctypes.c_void_p(1),
                     1, 1, None, 0, None)
    assert rc == 1 and b"iso_source" in lib.xr_last_error()
    ok = _native.geom3d_from_values(vals)
    rc = lib.xr_dd3d(0, ctypes.byref(ok), ctypes.c_void_p(256), 0, ctypes.c_void_p(256), 0, ctypes.c_void_p(256),
                     1, 1, None, 0, None)
    assert rc == 2 and b"workspace" in lib.xr_last_error()
    rc = lib.xr_dd3d(9, ctypes.byref(ok), None, 0, None, 0, None, 1, 1, None, 0, None)
    assert rc == 1


def test_projection_staging_plans_without_gpu():
    """The host planner of the TMA projection (no GPU needed): the window box
    the 512x512x256 / 1024x256 cone-flat workload is launched with, the
    fine-row walk for rows shorter than a voxel and the general walk for rows
    longer than one."""
    opts = load_golden("options")
    c5 = _native.cell_plan(_native.geom3d_from_values(opts["c5_3d_flat"]))
    assert c5 == dict(ok=True, box_pixels=48, box_z=115, rows_per_thread=16, fine=True), c5
    c2 = _native.cell_plan(_native.geom3d_from_values(opts["c2_3d_flat"]))
    assert c2["ok"] and c2["box_pixels"] % 8 == 0 and c2["rows_per_thread"] == 8
    coarse = _native.cell_plan(_native.geom3d_from_values(
        G.pack_options3d(G.Volume3d((64, 64, 24), 1.0), G.ConeBeam3d(G.Detector3d((40, 12), 2.5), 300., 600., "flat"))))
    assert coarse["ok"] and not coarse["fine"], coarse
    # the plan is a pure function of the geometry
    assert _native.cell_plan(_native.geom3d_from_values(opts["c5_3d_flat"])) == c5


def test_backprojection_staging_plans_without_gpu():
    """The host planner of the staged prefix backprojection (no GPU needed):
    the table box of the 512x512x256 / 1024x256 cone-flat workload is capped
    at two stages for four CTAs per SM (the few larger windows go to the
    fallback launch); parallel and arc geometries are planned too, odd
    column counts are not."""
    opts = load_golden("options")
    c5 = _native.pfx_stage_plan(_native.geom3d_from_values(opts["c5_3d_flat"]))
    assert c5["ok"] and c5["box_cols"] % 2 == 0, c5
    smem = 2 * 64 * 16 + 128 + 2 * ((c5["box_cols"] * c5["box_rows"] * 8 + 127) // 128 * 128)
    assert 4 * (smem + 1024) <= 228 * 1024, (c5, smem)
    par = _native.pfx_stage_plan(_native.geom3d_from_values(
        G.pack_options3d(G.Volume3d((64, 64, 32), 1.0), G.ParallelBeam3d(G.Detector3d((96, 40), 1.0)))))
    assert par["ok"], par
    arc = _native.pfx_stage_plan(_native.geom3d_from_values(
        G.pack_options3d(G.Volume3d((64, 64, 32), 1.0), G.ConeBeam3d(G.Detector3d((96, 40), 1.0), 300., 600., "arc"))))
    odd = _native.pfx_stage_plan(_native.geom3d_from_values(
        G.pack_options3d(G.Volume3d((64, 64, 32), 1.0), G.ConeBeam3d(G.Detector3d((95, 40), 1.0), 300., 600., "flat"))))
    assert arc["ok"] and not odd["ok"], (arc, odd)
    assert _native.pfx_stage_plan(_native.geom3d_from_values(opts["c5_3d_flat"])) == c5


@pytest.mark.parametrize("case", ["arc4d", "flat5d", "arc5d_grid"])
def test_rebin_grid_matches_reference(case):
    """The rebinning's host-side grid (xrecon_b200.rebin.rebin_grid, float32
    torch arithmetic as rebin.py:67-95) on CPU tensors: the parallel bin
    centres equal the reference's bit for bit, and every sample coordinate
    of the grid is finite."""
    from xrecon_b200.rebin import rebin_grid
    g = load_golden(f"rebin_{case}")
    kw = {k[3:]: (g[k] if g[k].ndim else g[k].item()) for k in g if k.startswith("kw_")}
    Nu = g["sino"].shape[-1]
    ang = torch.from_numpy(g["angles"])
    out_ang = torch.from_numpy(np.asarray(kw.get("output_angles", g["angles"]), np.float32))
    Nt = int(kw.get("output_det_count", Nu))
    grid, t = rebin_grid(ang, Nu, float(g["iso_source"]), float(g["det_spacing"]), float(g["det_shift"]),
                         str(g["detector_type"]), out_ang, Nt, kw.get("output_det_spacing"),
                         float(kw.get("output_det_shift", 0.0)))
    np.testing.assert_array_equal(t.numpy(), g["t"])
    assert tuple(grid.shape) == (out_ang.numel(), Nt, 2) and torch.isfinite(grid).all()
    np.testing.assert_array_equal(out_ang.numpy(), g["out_angles"])


def test_cpu_tensors_are_rejected():
    P = Projector3d(G.Volume3d((8, 8, 4), 1.0), G.ConeBeam3d(G.Detector3d((12, 6), 1.5), 500., 1000., "flat"))
    with pytest.raises(RuntimeError, match="CUDA"):
        P.projection(torch.zeros(1, 1, 4, 8, 8), torch.zeros(3))


def test_backend_surface_matches_reference_names():
    from xrecon_b200 import backend
    names = ["forward_projection2d", "backward_projection2d", "weighted_backward_projection2d",
             "projection_transpose2d", "backward_projection_transpose2d",
             "weighted_backward_projection_transpose2d", "back_projection2d", "weighted_back_projection2d",
             "forward_projection3d", "projection_transpose3d", "backward_projection3d",
             "weighted_backward_projection3d", "backward_projection_transpose3d",
             "weighted_backward_projection_transpose3d"]
    for n in names:
        assert callable(getattr(backend, n))
    with pytest.raises(RuntimeError, match="at least 18"):
        backend._geom(3, torch.zeros(10))


HELICAL_CASES = {
    "one_turn": dict(image_size=(32, 32, 16), num_det=(48, 8), pix_size=(2.0, 2.0, 1.0), det_size=(2.4, 2.0),
                     iso_source=300.0, source_detector=600.0, pixshift=(0.1, -0.2, 0.3), binshift=(0.3, -0.1),
                     pitch=8.0, z0=-8.0),
    "auto_tang": dict(image_size=(24, 20, 12), num_det=(40, 6), pix_size=(2.5, 2.5, 1.5), det_size=(3.0, 2.5),
                      iso_source=320.0, source_detector=640.0, pitch=12.0, z0=-9.0, helical_view_mode="auto",
                      helical_weight_mode="tang3d", helical_tang_k=3.0, helical_tang_blend=0.6, filter_type="hann"),
    "half_scan": dict(image_size=(32, 32, 16), num_det=(48, 8), pix_size=(2.0, 2.0, 1.0), det_size=(2.4, 2.0),
                      iso_source=300.0, source_detector=600.0, pitch=14.0, z0=-10.0, helical_view_mode="half",
                      helical_halfscan_coef=1.1, filter_type="shepplogan"),
}


@pytest.mark.parametrize("case", sorted(HELICAL_CASES))
def test_helical_projector_host_tables_match_reference(case):
    """Packed options, cell weight, filter, source positions and mean angle
    step of HelicalProjector3d against the reference's own class
    (tests/golden/helical_host.npz)."""
    from xrecon_b200 import HelicalProjector3d
    g = load_golden("helical_host")
    P = HelicalProjector3d(**HELICAL_CASES[case])
    np.testing.assert_array_equal(P.options.numpy(), g[f"{case}_options"])
    np.testing.assert_allclose(P.weight.numpy(), g[f"{case}_weight"], rtol=1e-6, atol=0)
    ref_f = g[f"{case}_filter"]
    np.testing.assert_allclose(P.filter.numpy(), ref_f, rtol=2e-6, atol=1e-7 * np.abs(ref_f).max())
    ang = torch.from_numpy(g[f"{case}_angles"])
    np.testing.assert_allclose(P.source_position(ang).numpy(), g[f"{case}_source_pos"], rtol=1e-6, atol=1e-6)
    assert abs(float(P._mean_angle_step(ang)) - float(g[f"{case}_mean_step"])) <= 1e-7


def test_helical_validation_without_gpu():
    """xr_helical3d argument checks (no kernel runs): arc detector only,
    known view / weight modes, workspace size."""
    from xrecon_b200 import HelicalProjector3d, backend
    P = HelicalProjector3d(**HELICAL_CASES["one_turn"])
    lib = _native.lib()
    g = P._host_geom.struct
    h = P._host_geom.hopts
    assert (h.view_mode, h.weight_mode) == (2, 0)
    for op in range(6):
        assert lib.xr_helical3d_workspace_size(op, ctypes.byref(g), 1, 192) > 0
    p = ctypes.c_void_p(256)
    flat = _native.geom3d_from_values(P.options.tolist()[:17] + [1.0])
    rc = lib.xr_helical3d(0, ctypes.byref(flat), ctypes.byref(h), p, p, p, p, 1, 4, None, 0, None)
    assert rc == 1 and b"arc" in lib.xr_last_error()
    bad = _native.HelicalOpts(view_mode=7, weight_mode=0, view_turns=0.0, halfscan_coef=1.0, tang_k=5.0,
                              tang_blend=0.0)
    rc = lib.xr_helical3d(0, ctypes.byref(g), ctypes.byref(bad), p, p, p, p, 1, 4, None, 0, None)
    assert rc == 1 and b"view mode" in lib.xr_last_error()
    rc = lib.xr_helical3d(4, ctypes.byref(g), ctypes.byref(h), p, p, p, p, 1, 4, None, 0, None)
    assert rc == 2 and b"workspace" in lib.xr_last_error()
    for n in ("forward_projection_helical3d", "projection_transpose_helical3d", "backward_projection_helical3d",
              "weighted_backward_projection_helical3d", "backward_projection_transpose_helical3d",
              "weighted_backward_projection_transpose_helical3d"):
        assert callable(getattr(backend, n))
    with pytest.raises(NotImplementedError):
        HelicalProjector3d(**dict(HELICAL_CASES["one_turn"], scan_type="flat"))
    with pytest.raises(ValueError, match="helical_view_mode"):
        HelicalProjector3d(**dict(HELICAL_CASES["one_turn"], helical_view_mode="spiral"))
    with pytest.raises(RuntimeError, match="CUDA"):
        P.projection(torch.zeros(1, 1, 16, 32, 32), torch.zeros(3))


def test_helical_projector_object_constructor_matches_legacy():
    """HelicalProjector3d(Volume3d, HelicalConeBeam3d) packs the same options
    as the legacy keyword form (projector3d.py:323-345)."""
    from xrecon_b200 import Detector3d, HelicalConeBeam3d, HelicalProjector3d, Volume3d
    kw = HELICAL_CASES["one_turn"]
    legacy = HelicalProjector3d(**kw)
    vol = Volume3d(kw["image_size"], kw["pix_size"], kw["pixshift"])
    geo = HelicalConeBeam3d(Detector3d(kw["num_det"], kw["det_size"], kw["binshift"]), kw["iso_source"],
                            kw["source_detector"], "arc", pitch=kw["pitch"], z0=kw["z0"])
    obj = HelicalProjector3d(vol, geo)
    np.testing.assert_array_equal(obj.options.numpy(), legacy.options.numpy())
    assert (obj.pitch, obj.z0) == (8.0, -8.0)
    with pytest.raises(TypeError):
        HelicalProjector3d(vol, Detector3d(kw["num_det"], kw["det_size"]))
