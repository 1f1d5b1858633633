"""Parity of the CUDA operators (through the C ABI) with the FP64 oracle and
with the reference's own outputs.

Tolerances (relative L2):
* against the FP64 oracle: 1e-5 (the parity bar for FP32); for the arc
  detector the oracle takes the CUDA path's float32 boundary arithmetic
  (tests/conftest.py), which differs from the reference's only where the C
  library's tanf is off by one unit;
* against the reference fixtures: 1e-5 for every geometry, arc included;
* adjoint pairs <Ax, y> = <x, A^T y>: 1e-5;
* BF16/FP16 storage with FP32 accumulation: 1e-3 against the oracle applied
  to the same (rounded) input; outputs stored in BF16 add their own rounding
  (2^-9 relative RMS), bounded at 3e-3.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OPS = ("A", "AT", "B", "BT", "BW", "BWT")
IMG_IN = ("A", "BT", "BWT")


def run(dim, op, x, options, angles, dev, dtype=torch.float32, out_dtype=None):
    from xrecon_b200 import _native
    from xrecon_b200.backend import HostGeometry
    g = HostGeometry(dim, np.asarray(options).tolist()).struct
    xt = torch.as_tensor(np.ascontiguousarray(x)).to(device=dev, dtype=dtype)
    at = torch.as_tensor(np.asarray(angles, np.float32)).to(dev)
    y = _native.apply(dim, op, xt, g, at, out_dtype=out_dtype)
    torch.cuda.synchronize()
    return y.float().cpu().numpy()


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_ops_match_oracle_and_reference(cuda, dim, scan):
    g = load_golden(f"dd{dim}d_{scan}")
    ofn = O.dd2d if dim == 2 else O.dd3d
    for op in OPS:
        x = g["image"] if op in IMG_IN else g["sino"]
        got = run(dim, op, x, g["options"], g["angles"], cuda)
        exact = ofn(op, x, g["options"], g["angles"])
        e_oracle = rel_l2(got, exact)
        assert e_oracle < 1e-5, f"{dim}D {scan} {op}: vs oracle {e_oracle:.2e}"
        e_ref = rel_l2(got, g[op])
        assert e_ref < 1e-5, f"{dim}D {scan} {op}: vs reference {e_ref:.2e}"


def _opts3d(W, H, D, Nu, Nv, dx, dy, dz, du, dv, sod, sdd, sh, shu, shv, scan):
    from xrecon_b200 import geometry as G
    det = G.Detector3d((Nu, Nv), (du, dv), (shu, shv))
    geo = G.ParallelBeam3d(det) if scan == "parallel" else G.ConeBeam3d(det, sod, sdd, scan)
    return np.array(G.pack_options3d(G.Volume3d((W, H, D), (dx, dy, dz), sh), geo), np.float32)


def _opts2d(W, H, Nu, dx, dy, du, sod, sdd, sh, shu, scan):
    from xrecon_b200 import geometry as G
    det = G.Detector2d(Nu, du, shu)
    geo = G.ParallelBeam2d(det) if scan == "parallel" else G.FanBeam2d(det, sod, sdd, scan)
    return np.array(G.pack_options2d(G.Volume2d((W, H), (dx, dy), sh), geo), np.float32)


@pytest.mark.parametrize("scan", ["flat", "arc", "parallel"])
def test_config2_shapes_against_oracle(cuda, scan):
    """256x256x64 volume, 384x96 detector (config 2 geometry) on a subset of
    views including the 45-degree axis switches, random (worst-case) data."""
    opts = _opts3d(256, 256, 64, 384, 96, 1.0, 1.0, 1.0, 1.5, 1.5, 500., 1000., 0.0, 0.0, 0.0, scan)
    ang = (np.array([3, 90, 180, 270, 500, 719]) * (2 * np.pi / 720)).astype(np.float32)
    rng = np.random.default_rng(2)
    img = rng.random((1, 1, 64, 256, 256)).astype(np.float32)
    sino = rng.random((1, 1, ang.size, 96, 384)).astype(np.float32)
    for op in ("A", "B", "AT", "BWT"):
        x = img if op in IMG_IN else sino
        got = run(3, op, x, opts, ang, cuda)
        exact = O.dd3d(op, x, opts, ang)
        assert rel_l2(got, exact) < 1e-5, (scan, op)


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_adjoint_dot_products(cuda, dim, scan):
    if dim == 3:
        opts = _opts3d(33, 29, 17, 45, 21, 1.0, 0.9, 1.1, 1.3, 1.2, 400., 800., (0.4, -0.3, 0.2), 0.3, -0.2, scan)
    else:
        opts = _opts2d(61, 47, 77, 0.9, 1.1, 1.3, 400., 800., (0.4, -0.3), 0.3, scan)
    ang = (np.arange(40) * (2 * np.pi / 40) + 0.05).astype(np.float32)
    # non-negative data: the dot products carry no cancellation, so their
    # relative difference measures the operators, not the summation order
    rng = np.random.default_rng(3)
    if dim == 3:
        x = rng.random((1, 1, 17, 29, 33)).astype(np.float32)
        y = rng.random((1, 1, 40, 21, 45)).astype(np.float32)
    else:
        x = rng.random((1, 1, 47, 61)).astype(np.float32)
        y = rng.random((1, 1, 40, 77)).astype(np.float32)
    for fwd, adj in (("A", "AT"), ("BT", "B"), ("BWT", "BW")):
        lhs = float(np.sum(run(dim, fwd, x, opts, ang, cuda).astype(np.float64) * y))
        rhs = float(np.sum(x.astype(np.float64) * run(dim, adj, y, opts, ang, cuda)))
        assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs)) / 2, (fwd, adj, lhs, rhs)


def test_deterministic_and_batched(cuda):
    g = load_golden("dd3d_flat")
    rng = np.random.default_rng(4)
    img = rng.random((2, 3) + g["image"].shape[2:]).astype(np.float32)
    sino = rng.random((2, 3) + g["sino"].shape[2:]).astype(np.float32)
    for op in OPS:
        x = img if op in IMG_IN else sino
        a = run(3, op, x, g["options"], g["angles"], cuda)
        b = run(3, op, x, g["options"], g["angles"], cuda)
        assert np.array_equal(a, b), f"{op} not bitwise reproducible"
        one = run(3, op, x[1:2, 2:3], g["options"], g["angles"], cuda)
        assert np.array_equal(a[1:2, 2:3], one), f"{op}: batch element differs from single call"


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_half_storage_forms(cuda, dtype):
    g = load_golden("dd3d_flat")
    for op in OPS:
        x = g["image"] if op in IMG_IN else g["sino"]
        xq = torch.as_tensor(x).to(dtype).float().numpy()  # what the kernel sees
        exact = O.dd3d(op, xq, g["options"], g["angles"])
        got32 = run(3, op, x, g["options"], g["angles"], cuda, dtype=dtype, out_dtype=torch.float32)
        assert rel_l2(got32, exact) < 1e-5, (dtype, op, "fp32 accumulation")
        goth = run(3, op, x, g["options"], g["angles"], cuda, dtype=dtype)
        bound = 3e-3 if dtype == torch.bfloat16 else 1e-3
        assert rel_l2(goth, exact) < bound, (dtype, op, "half output")


def test_edges_odd_shapes_and_empty(cuda):
    # detector narrower than the volume, strong shifts, Nu not a multiple of 32
    opts = _opts3d(20, 37, 9, 7, 5, 1.0, 1.0, 1.0, 2.5, 2.5, 300., 700., (3.0, -2.0, 1.5), 1.5, -1.0, "flat")
    ang = np.array([0.0, 0.3, 1.2, 2.5, 3.9, 5.5], np.float32)
    rng = np.random.default_rng(5)
    img = rng.random((1, 1, 9, 37, 20)).astype(np.float32)
    sino = rng.random((1, 1, 6, 5, 7)).astype(np.float32)
    for op in OPS:
        x = img if op in IMG_IN else sino
        assert rel_l2(run(3, op, x, opts, ang, cuda), O.dd3d(op, x, opts, ang)) < 1e-5, op
    # zero views: volume outputs are zero, sinogram outputs empty
    empty = np.zeros(0, np.float32)
    assert np.all(run(3, "B", np.zeros((1, 1, 0, 5, 7), np.float32), opts, empty, cuda) == 0)
    assert run(3, "A", img, opts, empty, cuda).shape == (1, 1, 0, 5, 7)


@pytest.mark.parametrize("scan", ["flat", "arc", "parallel"])
def test_tma_and_plain_paths_match_oracle(cuda, scan):
    """The staged kernels (TMA line windows for A/B^T/Bw^T, row prefix tables
    for A^T/B/Bw) and the plain kernels both match the oracle (windows clamped
    at the image edges, detector wider and narrower than the image, rows
    finer and coarser than voxels, shifted geometries)."""
    from xrecon_b200 import _native
    cases = [
        _opts3d(96, 80, 40, 128, 48, 1.0, 1.0, 1.0, 1.2, 1.2, 400., 800., (0.5, -0.3, 0.7), 0.3, -0.4, scan),
        _opts3d(64, 64, 24, 40, 12, 1.0, 1.0, 1.0, 2.5, 2.5, 300., 600., (4.0, -3.0, 2.0), 1.5, -1.0, scan),
        _opts3d(50, 70, 130, 96, 160, 1.0, 1.0, 1.0, 1.0, 1.0, 500., 900., 0.0, 0.0, 0.0, scan),
    ]
    ang = (np.arange(0, 24) * (2 * np.pi / 24) + 0.02).astype(np.float32)
    ang = np.concatenate([ang, np.array([np.pi / 4, 3 * np.pi / 4], np.float32)])
    rng = np.random.default_rng(9)
    if scan != "parallel":
        # both projection kernels are exercised: rows finer than voxels in the
        # first case, coarser in the second
        plans = [_native.cell_plan(_native.geom3d_from_values(o.tolist())) for o in cases]
        assert plans[0]["fine"] and not plans[1]["fine"], plans
    try:
        for opts in cases:
            D, H, W = int(opts[2]), int(opts[1]), int(opts[0])
            img = rng.random((1, 1, D, H, W)).astype(np.float32)
            sino = rng.random((1, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
            for op in ("A", "BT", "BWT", "AT", "B", "BW"):
                x = img if op in ("A", "BT", "BWT") else sino
                exact = O.dd3d(op, x, opts, ang)
                _native.set_plain_kernels(False)
                tma = run(3, op, x, opts, ang, cuda)
                _native.set_plain_kernels(True)
                plain = run(3, op, x, opts, ang, cuda)
                assert rel_l2(tma, exact) < 1e-5, (scan, op, "tma")
                assert rel_l2(plain, exact) < 1e-5, (scan, op, "plain")
    finally:
        _native.set_plain_kernels(False)


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
def test_backprojection_deep_volumes(cuda, scan):
    """B, Bw and A^T against the oracle on volumes 640 and 900 slices deep
    (one shifted 300 mm along z, with a detector offset along v): the prefix
    gather evaluates each (pixel, view)'s first column in FP64 and the next
    columns' run offsets as that value plus z times the change of rows per
    voxel in FP32, which grows with the run's distance from z = 0."""
    cases = [
        _opts3d(12, 10, 640, 48, 800, 1.0, 1.0, 1.0, 1.1, 1.0, 500., 1000., (0.5, -0.3, 0.0), 0.2, 0.3, scan),
        _opts3d(10, 12, 900, 40, 700, 1.2, 1.1, 0.8, 1.4, 1.6, 450., 900., (0.2, 0.4, 300.0), -0.3, 120.0, scan),
    ]
    ang = (np.arange(16) * (2 * np.pi / 16) + 0.07).astype(np.float32)
    rng = np.random.default_rng(21)
    for opts in cases:
        sino = rng.random((1, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
        for op in ("B", "BW", "AT"):
            got = run(3, op, sino, opts, ang, cuda)
            assert rel_l2(got, O.dd3d(op, sino, opts, ang)) < 1e-5, (scan, op)


@pytest.mark.parametrize("scan", ["flat", "arc", "parallel"])
def test_backprojection_long_column_walks(cuda, scan):
    """B, Bw and A^T (prefix-table and plain gathers) against the oracle when
    pixels are much wider than the detector cells: pixels of 4 mm over cells
    of 0.5 mm put about 16 columns on every pixel (long column walks; on the
    arc detector, chains that drift several float units from the direct
    angles); 40 x 44 pixels leave partial CTA tiles at both edges; the second
    geometry has pixels finer than cells."""
    from xrecon_b200 import _native
    cases = [
        _opts3d(40, 44, 20, 600, 24, 4.0, 4.0, 1.0, 0.5, 1.0, 500., 1000., (1.0, -2.0, 0.5), 0.2, 0.1, scan),
        _opts3d(72, 56, 33, 40, 20, 0.5, 0.5, 0.6, 2.0, 2.0, 400., 800., (0.3, 0.2, -0.4), -0.5, 0.3, scan),
    ]
    ang = np.concatenate([(np.arange(12) * (2 * np.pi / 12) + 0.1), [np.pi / 4, 3 * np.pi / 4]]).astype(np.float32)
    rng = np.random.default_rng(11)
    try:
        for opts in cases:
            sino = rng.random((1, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
            for op in ("B", "BW", "AT"):
                exact = O.dd3d(op, sino, opts, ang)
                _native.set_plain_kernels(False)
                staged = run(3, op, sino, opts, ang, cuda)
                _native.set_plain_kernels(True)
                plain = run(3, op, sino, opts, ang, cuda)
                assert rel_l2(staged, exact) < 1e-5, (scan, op, "prefix tables")
                assert rel_l2(plain, exact) < 1e-5, (scan, op, "plain")
    finally:
        _native.set_plain_kernels(False)
