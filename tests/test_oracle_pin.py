"""Pin the FP64 oracle against the reference's own outputs (CPU only).

The golden fixtures hold outputs of the reference's CPU path (its Python
package over its C++ CPU kernels, see tests/golden/make_golden.py).  The
reference computes its geometry in float32; its distance from the exact
operator is ~1e-6 (relative L2) for parallel and flat geometries at these
sizes and up to ~1.5e-4 for the arc geometry, whose boundary angles
(k - Nu/2)*du + shift_u + beta are rounded to float32 (a quantum of 4.8e-7 rad
at |beta| ~ 2 pi, up to 5e-4 of a detector cell), mapped to the axis in float
(src.x + src.y tanf(a) cancels to about ulp(|src|)) and, in the voxel-driven
operators, chained from column to column.  The oracle restates those three
roundings for the circular arc detector (dd_oracle.c arc_angle, map_angle_f,
chain_overlaps), so every geometry is held to 1e-5; arc_exact=True gives the
exact operator.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import oracle as O

OPS = ("A", "AT", "B", "BT", "BW", "BWT")
IMG_IN = ("A", "BT", "BWT")
TOL = {"parallel": 1e-5, "flat": 1e-5, "arc": 1e-5}


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_matches_reference_outputs(dim, scan):
    g = load_golden(f"dd{dim}d_{scan}")
    fn = O.dd2d if dim == 2 else O.dd3d
    for op in OPS:
        x = g["image"] if op in IMG_IN else g["sino"]
        got = fn(op, x, g["options"], g["angles"])
        err = rel_l2(got, g[op])
        assert err < TOL[scan], f"{dim}D {scan} {op}: rel L2 {err:.3e}"


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_adjoint_pairs(dim, scan):
    """<Ax, y> = <x, A^T y> and the same for B and Bw, in FP64."""
    g = load_golden(f"dd{dim}d_{scan}")
    fn = O.dd2d if dim == 2 else O.dd3d
    x, y = g["image"].astype(np.float64), g["sino"].astype(np.float64)
    for fwd, adj in (("A", "AT"), ("BT", "B"), ("BWT", "BW")):
        lhs = float(np.sum(fn(fwd, x, g["options"], g["angles"]) * y))
        rhs = float(np.sum(x * fn(adj, y, g["options"], g["angles"])))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (fwd, adj, lhs, rhs)


@pytest.mark.parametrize("case", ["flat_ramp", "arc_ramp", "parallel_shepplogan", "flat_hann", "flat_parker"])
def test_oracle_fbp_matches_reference(case):
    g = load_golden(f"fbp2d_{case}")
    redundant = case != "flat_parker"
    parker = g["parker"].reshape(1, 1, g["angles"].size, -1) if g["parker"].size else None
    got = O.filtered_backprojection2d(g["sino"], g["options"], g["angles"], g["weight"], g["filter"],
                                      redundant=redundant, parker=parker)
    assert rel_l2(got, g["recon"]) < 2e-5


@pytest.mark.parametrize("case", ["flat", "arc"])
def test_oracle_fdk_matches_reference(case):
    g = load_golden(f"fdk3d_{case}")
    got = O.filtered_backprojection3d(g["sino"], g["options"], g["angles"], g["weight"], g["filter"])
    assert rel_l2(got, g["recon"]) < 2e-5


ADJOINT = {"A": "AT", "AT": "A", "B": "BT", "BT": "B", "BW": "BWT", "BWT": "BW"}


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_transposes_are_the_reference_autograd_gradients(dim, scan):
    """The gradients the reference's own autograd Functions return (their
    backward is the partner transpose binding, functions.py:96-302; fixtures
    from tests/golden/make_golden.py autograd) equal the oracle's transposes
    of the upstream gradient.  The CUDA Functions' backward is checked
    against the same oracle transposes on the GPU."""
    g = load_golden(f"autograd{dim}d_{scan}")
    fn = O.dd2d if dim == 2 else O.dd3d
    for op, adj in ADJOINT.items():
        assert g[f"{op}_grad"].shape == g[f"{op}_x"].shape
        exact = fn(adj, g[f"{op}_u"], g["options"], g["angles"])
        assert rel_l2(g[f"{op}_grad"], exact) < TOL[scan], (op, adj)


def test_oracle_reference_library_when_present():
    """Where oracle/_ref was built, run a fresh seeded case through both."""
    from oracle import refcpu
    if not refcpu.available():
        pytest.skip("reference CPU library not built")
    g = load_golden("dd3d_flat")
    rng = np.random.default_rng(7)
    x = rng.random(g["image"].shape).astype(np.float32)
    a = O.dd3d("A", x, g["options"], g["angles"])
    b = refcpu.dd3d("A", x, g["options"], g["angles"])
    assert rel_l2(b, a) < 1e-5


def _random_case(rng, dim, scan):
    """A seeded small geometry: odd sizes, anisotropic spacings, volume and
    detector shifts, source outside the volume, random angles plus two on
    the 45-degree axis switch; random image and sinogram."""
    from xrecon_b200 import geometry as G
    W, H = (int(v) for v in rng.integers(8, 33, 2))
    D, Nu, Nv, V = int(rng.integers(4, 13)), int(rng.integers(8, 49)), int(rng.integers(4, 17)), int(rng.integers(4, 13))
    dx, dy, dz = rng.uniform(0.6, 1.6, 3)
    du, dv = rng.uniform(0.8, 2.0, 2)
    sod = rng.uniform(300, 600)
    sdd = sod * rng.uniform(1.5, 2.5)
    sh = tuple(rng.uniform(-3, 3, 3))
    shu, shv = rng.uniform(-2, 2, 2)
    ang = np.concatenate([rng.uniform(0, 2 * np.pi, V), [np.pi / 4, 5 * np.pi / 4]]).astype(np.float32)
    if dim == 3:
        det = G.Detector3d((Nu, Nv), (du, dv), (shu, shv))
        geo = G.ParallelBeam3d(det) if scan == "parallel" else G.ConeBeam3d(det, sod, sdd, scan)
        o = np.array(G.pack_options3d(G.Volume3d((W, H, D), (dx, dy, dz), sh), geo), np.float32)
        img, sino = rng.random((1, 1, D, H, W)), rng.random((1, 1, ang.size, Nv, Nu))
    else:
        det = G.Detector2d(Nu, du, shu)
        geo = G.ParallelBeam2d(det) if scan == "parallel" else G.FanBeam2d(det, sod, sdd, scan)
        o = np.array(G.pack_options2d(G.Volume2d((W, H), (dx, dy), sh[:2]), geo), np.float32)
        img, sino = rng.random((1, 1, H, W)), rng.random((1, 1, ang.size, Nu))
    return o, ang, img.astype(np.float32), sino.astype(np.float32)


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_matches_reference_library_on_random_geometries(dim, scan):
    """Where oracle/_ref was built: 40 seeded random geometries, all six
    operators, the oracle against the reference's own CPU kernels, within the
    reference's float32-geometry distance (TOL)."""
    from oracle import refcpu
    if not refcpu.available():
        pytest.skip("reference CPU library not built")
    f, g = (O.dd2d, refcpu.dd2d) if dim == 2 else (O.dd3d, refcpu.dd3d)
    for seed in range(40):
        o, ang, img, sino = _random_case(np.random.default_rng(1000 + seed), dim, scan)
        for op in OPS:
            x = img if op in IMG_IN else sino
            exact = f(op, x, o, ang)
            assert np.linalg.norm(exact) > 0, (seed, op)
            assert rel_l2(g(op, x, o, ang), exact) < TOL[scan], (seed, op)


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_adjoint_pairs_on_random_geometries(dim, scan):
    """The oracle's transposes are exact adjoints (FP64) on 20 seeded random
    geometries per dimension and scan type, not only on the fixtures'."""
    fn = O.dd2d if dim == 2 else O.dd3d
    for seed in range(20):
        o, ang, img, sino = _random_case(np.random.default_rng(2000 + seed), dim, scan)
        x, y = img.astype(np.float64), sino.astype(np.float64)
        for fwd, adj in (("A", "AT"), ("BT", "B"), ("BWT", "BW")):
            lhs = float(np.sum(fn(fwd, x, o, ang) * y))
            rhs = float(np.sum(x * fn(adj, y, o, ang)))
            assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (seed, fwd, adj, lhs, rhs)


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_reference_system_matrix_is_the_oracle_projection(dim, scan):
    """The reference's sparse projection matrix (fixture) times an image is
    the oracle's projection: pins the matrix conventions (rows: view, detector
    row, physical column; columns: flattened voxels)."""
    g = load_golden(f"sysmat{dim}d_{scan}")
    shape = tuple(int(s) for s in g["shape"])
    M = np.zeros(shape)
    np.add.at(M, (g["rows"], g["cols"]), g["vals"])
    rng = np.random.default_rng(4)
    o = g["options"]
    img_shape = (1, 1, int(o[1]), int(o[0])) if dim == 2 else (1, 1, int(o[2]), int(o[1]), int(o[0]))
    x = rng.random(img_shape)
    exact = (O.dd2d if dim == 2 else O.dd3d)("A", x, o, g["angles"]).reshape(-1)
    assert rel_l2(M @ x.reshape(-1), exact) < TOL[scan]


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_reference_system_matrix_on_random_geometries(dim, scan):
    """Where oracle/_ref was built: the reference's own sparse projection
    matrix (system_matrix2d/3d CPU code) times a random image equals the
    oracle's projection on 10 seeded random geometries per dimension and
    scan type."""
    from oracle import refcpu
    if not refcpu.available():
        pytest.skip("reference CPU library not built")
    fn = O.dd2d if dim == 2 else O.dd3d
    for seed in range(10):
        o, ang, img, _ = _random_case(np.random.default_rng(3000 + seed), dim, scan)
        rows, cols, vals, shape = refcpu.system_matrix(dim, o, ang)
        y = np.zeros(shape[0])
        np.add.at(y, rows, vals.astype(np.float64) * img.reshape(-1)[cols])
        exact = fn("A", img, o, ang).reshape(-1)
        assert rel_l2(y, exact) < TOL[scan], seed


def _rebin_kwargs(g):
    kw = {}
    for k in g:
        if k.startswith("kw_"):
            v = g[k]
            kw[k[3:]] = v if v.ndim else v.item()
    return kw


@pytest.mark.parametrize("case", ["arc4d", "flat5d", "arc5d_grid"])
def test_oracle_rebin_matches_reference(case):
    g = load_golden(f"rebin_{case}")
    out, oa, t = O.fan_to_parallel_rebin(g["sino"], g["angles"], float(g["iso_source"]), float(g["det_spacing"]),
                                         float(g["det_shift"]), str(g["detector_type"]), **_rebin_kwargs(g))
    assert out.shape == g["out"].shape
    np.testing.assert_array_equal(t, g["t"])
    assert rel_l2(out, g["out"]) < 1e-5


# ---------------------------------------------------------------- helical

def _helical_case():
    """Small arc geometry, 60 views over one turn, and its options vector."""
    W, H, D, Nu, Nv = 24, 24, 12, 40, 8
    opts = np.array([W, H, D, Nu, Nv, 1.0, 1.0, 1.0, 0.004, 1.2, 300.0, 600.0, 0.3, -0.2, 0.4, 0.001, 0.1, 2],
                    np.float32)
    V = 60
    ang = (np.arange(V) * (2 * np.pi / V) + 0.05).astype(np.float32)
    rng = np.random.default_rng(3)
    x = rng.random((1, 1, D, H, W))
    y = rng.random((1, 1, V, Nv, Nu))
    return opts, ang, x, y, rng


def test_helical_oracle_reduces_to_the_circular_arc():
    """With every source offset zero the helical operators are the cone-arc
    ones (which are pinned to the reference above): A and A^T identically, B
    and B^T up to the column width sod du vs 2 sod tan(du/2) (du^2/12).  With
    a constant source z, B and B^T equal the circular ones on a volume shifted
    by -z; A carries the reference's absolute-z cell cosine and moves."""
    opts, ang, x, y, _ = _helical_case()
    V = ang.size
    sp = np.zeros((4, V), np.float32)
    for op, inp, tol in (("A", x, 1e-12), ("AT", y, 1e-12), ("B", y, 2e-6), ("BT", x, 2e-6)):
        err = rel_l2(O.helical3d(op, inp, opts, ang, sp), O.dd3d(op, inp, opts, ang, arc_exact=True))
        assert err < tol, (op, err)
    c = np.float32(2.5)
    sp[0] = c
    shifted = opts.copy()
    shifted[14] = opts[14] - c
    for op, inp in (("B", y), ("BT", x)):
        assert rel_l2(O.helical3d(op, inp, opts, ang, sp), O.dd3d(op, inp, shifted, ang, arc_exact=True)) < 2e-6
    assert rel_l2(O.helical3d("A", x, opts, ang, sp), O.dd3d("A", x, shifted, ang, arc_exact=True)) > 1e-5


@pytest.mark.parametrize("modes", [(2, 0), (0, 1), (1, 0), (3, 0)])
def test_helical_oracle_adjoint_pairs(modes):
    """<A x, y> = <x, A^T y>, <B^T x, y> = <x, B y>, <Bw^T x, y> = <x, Bw y>
    with flying-focal-spot style offsets, for several view / weight modes."""
    opts, ang, x, y, rng = _helical_case()
    V = ang.size
    o = np.concatenate([opts, np.array([modes[0], modes[1], 1.5, 1.0, 4.0, 0.5], np.float32)])
    sp = np.zeros((4, V), np.float32)
    sp[0] = np.linspace(-4.0, 4.0, V)
    sp[1] = rng.normal(0.0, 1.0, V)
    sp[2] = rng.normal(0.0, 5e-4, V)
    sp[3] = rng.normal(0.0, 0.3, V)
    for fwd, adj in (("A", "AT"), ("BT", "B"), ("BWT", "BW")):
        lhs = float(np.sum(O.helical3d(fwd, x, o, ang, sp) * y))
        rhs = float(np.sum(x * O.helical3d(adj, y, o, ang, sp)))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (fwd, adj, lhs, rhs)
        assert lhs != 0.0


HELICAL_REF_TOL = {"A": 2e-4, "AT": 2e-4, "B": 2e-4, "BT": 2e-4, "BW": 5e-4, "BWT": 5e-4}


@pytest.mark.parametrize("case", ["one_turn_ffs", "auto_tang", "half_scan"])
def test_helical_oracle_matches_reference_cuda_outputs(case):
    """The FP64 helical oracle against the reference's own helical CUDA
    kernels (helical_arc3d.cu, built from its sources and run on a B200 by
    tests/golden/make_golden_helical.py).  The reference computes in FP32
    with --use_fast_math: measured distances are 1e-5 .. 9e-5 for A, A^T, B,
    B^T and up to 2.2e-4 for the weighted pair, whose few outlying voxels sit
    on discrete tests (detector edge, window quality) that fast-math rounding
    flips.  In the one-turn case with 96 views per turn the window length
    ceil(2 pi / dbeta) has an exact integer quotient; the reference's
    approximate division came out one view longer, which the oracle's
    window_quotient_up reproduces (without it Bw differs by 5e-3)."""
    g = load_golden(f"helical_ref_{case}")
    assert bool(g["guard_ok"]), "the reference wrote outside its output while recording"
    tie = case == "one_turn_ffs"
    for op in ("A", "AT", "B", "BT", "BW", "BWT"):
        x = g["image"] if op in IMG_IN else g["sino"]
        got = O.helical3d(op, x, g["options"], g["angles"], g["source_pos"],
                          window_quotient_up=tie and op in ("BW", "BWT"))
        err = rel_l2(got, g[op])
        assert err < HELICAL_REF_TOL[op], f"{case} {op}: rel L2 {err:.3e}"
    if tie:
        exact = O.helical3d("BW", g["sino"], g["options"], g["angles"], g["source_pos"])
        assert rel_l2(exact, g["BW"]) > 1e-3  # the tie is real: the exact window differs by a view
