"""Helical arc-detector operators (HelicalProjector3d) on the GPU against the
FP64 helical oracle (oracle/dd_oracle.c, xo_helical3d): the six operators for
several view / weight modes and flying-focal-spot offsets, adjointness of
the three pairs, the autograd pairing, helical FDK, the plain-kernel path and
edge cases (one view, two views, no views, batches)."""
import math

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OPS = ("A", "AT", "B", "BT", "BW", "BWT")
IMG_IN = ("A", "BT", "BWT")
METHOD = {"A": "projection", "AT": "projection_t", "B": "backprojection", "BT": "backprojection_t",
          "BW": "backprojection_weighted", "BWT": "backprojection_weighted_t"}
# FP32 accumulation against the FP64 oracle
TOL = 1e-5


def _projector(**over):
    from xrecon_b200 import HelicalProjector3d
    kw = dict(image_size=(32, 28, 16), num_det=(64, 8), pix_size=(1.5, 1.5, 1.0), det_size=(3.0, 2.0),
              iso_source=300.0, source_detector=600.0, pixshift=(0.2, -0.3, 0.25), binshift=(0.25, -0.1),
              pitch=8.0, z0=-9.0)
    kw.update(over)
    return HelicalProjector3d(**kw)


def _angles(V, per_turn=96, start=0.05):
    return (np.arange(V) * (2 * np.pi / per_turn) + start).astype(np.float32)


def _case_angles(case, V):
    """Increasing angles, or for the reverse case the same set walked
    downwards from 2.5 turns."""
    if case == "reverse":
        return (5 * np.pi - np.arange(V) * (2 * np.pi / 96)).astype(np.float32)
    return _angles(V)


CASES = {
    "one_turn": (dict(), False),
    "ffs": (dict(), True),
    "auto_tang": (dict(helical_view_mode="auto", helical_weight_mode="tang3d", helical_tang_k=3.0,
                       helical_tang_blend=0.6), True),
    "half_scan": (dict(helical_view_mode="half", helical_halfscan_coef=1.1, pitch=12.0, z0=-12.0), False),
    "turns": (dict(helical_view_mode="turns", helical_view_turns=1.5, pitch=6.0, z0=-9.0), False),
    # decreasing angles (negative angle step): the source still rises by
    # pitch per turn of |beta|, through z0 + pitch (beta - beta_0) / (2 pi)
    "reverse": (dict(pitch=-8.0, z0=-9.0), True),
}


def _source_pos(P, ang, ffs, seed=5):
    sp = P.source_position(torch.from_numpy(ang)).numpy().copy()
    if ffs:
        rng = np.random.default_rng(seed)
        V = ang.size
        sp[1] = rng.normal(0.0, 1.0, V)
        sp[2] = rng.normal(0.0, 5e-4, V)
        sp[3] = rng.normal(0.0, 0.3, V)
    return sp.astype(np.float32)


def _inputs(P, V, seed=11, batch=1):
    W, H, D = P.image_size
    Nu, Nv = P.num_det
    rng = np.random.default_rng(seed)
    x = rng.random((batch, 1, D, H, W)).astype(np.float32)
    y = rng.random((batch, 1, V, Nv, Nu)).astype(np.float32)
    return x, y


@pytest.mark.parametrize("case", sorted(CASES))
def test_helical_operators_match_oracle(cuda, case):
    over, ffs = CASES[case]
    P = _projector(**over)
    V = 240
    ang = _case_angles(case, V)
    sp = _source_pos(P, ang, ffs)
    x, y = _inputs(P, V)
    opts = P.options.numpy()
    a, s = torch.from_numpy(ang).to(cuda), torch.from_numpy(sp).to(cuda)
    for op in OPS:
        inp = x if op in IMG_IN else y
        got = getattr(P, METHOD[op])(torch.from_numpy(inp).to(cuda), a, s).cpu().numpy()
        ref = O.helical3d(op, inp, opts, ang, sp)
        assert np.linalg.norm(ref) > 0, op
        err = rel_l2(got, ref)
        assert err < TOL, f"{case} {op}: rel L2 {err:.3e}"


@pytest.mark.parametrize("case", ["ffs", "half_scan"])
def test_helical_adjoint_pairs(cuda, case):
    over, ffs = CASES[case]
    P = _projector(**over)
    V = 240
    ang = _angles(V)
    sp = _source_pos(P, ang, ffs, seed=9)
    x, y = _inputs(P, V, seed=13)
    a, s = torch.from_numpy(ang).to(cuda), torch.from_numpy(sp).to(cuda)
    xt, yt = torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda)
    for fwd, adj in (("A", "AT"), ("BT", "B"), ("BWT", "BW")):
        lhs = float((getattr(P, METHOD[fwd])(xt, a, s).double() * yt.double()).sum())
        rhs = float((xt.double() * getattr(P, METHOD[adj])(yt, a, s).double()).sum())
        assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (fwd, adj, lhs, rhs)


def test_helical_plain_kernels_match_oracle(cuda):
    """A, B^T and Bw^T through the plain (non-TMA) cell gathers."""
    from xrecon_b200 import _native
    P = _projector()
    V = 192
    ang = _angles(V)
    sp = _source_pos(P, ang, True, seed=3)
    x, _ = _inputs(P, V)
    a, s = torch.from_numpy(ang).to(cuda), torch.from_numpy(sp).to(cuda)
    _native.set_plain_kernels(True)
    try:
        for op in ("A", "BT", "BWT"):
            got = getattr(P, METHOD[op])(torch.from_numpy(x).to(cuda), a, s).cpu().numpy()
            assert rel_l2(got, O.helical3d(op, x, P.options.numpy(), ang, sp)) < TOL, op
    finally:
        _native.set_plain_kernels(False)


def test_helical_autograd_pairs(cuda):
    """Every helical Function's backward is its partner transpose
    (functions.py:305-388 of the reference)."""
    P = _projector()
    V = 144
    ang = torch.from_numpy(_angles(V)).to(cuda)
    x, y = _inputs(P, V, seed=4)
    xt, yt = torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda)
    pairs = (("projection", "projection_t", xt, yt), ("projection_t", "projection", yt, xt),
             ("backprojection", "backprojection_t", yt, xt), ("backprojection_t", "backprojection", xt, yt),
             ("backprojection_weighted", "backprojection_weighted_t", yt, xt),
             ("backprojection_weighted_t", "backprojection_weighted", xt, yt))
    for fwd, adj, inp, cot in pairs:
        v = inp.clone().requires_grad_(True)
        out = getattr(P, fwd)(v, ang)
        assert out.shape == cot.shape
        (out * cot).sum().backward()
        exp = getattr(P, adj)(cot, ang)
        assert torch.equal(v.grad, exp), fwd


def test_helical_fdk_matches_oracle(cuda):
    """filtered_backprojection = Bw(corr_u(sino * w, h)) * mean angle step
    (projector3d.py:465-481), fused filter path and differentiable path."""
    P = _projector()
    V = 240
    ang = _angles(V)
    sp = P.source_position(torch.from_numpy(ang)).numpy()
    _, y = _inputs(P, V, seed=21)
    a = torch.from_numpy(ang).to(cuda)
    rec = P.filtered_backprojection(torch.from_numpy(y).to(cuda), a).cpu().numpy()
    sw = y.astype(np.float64) * P.weight.numpy().astype(np.float64)
    filt = P.filter.numpy().reshape(-1)
    filtered = O.correlate_rows(sw, filt)
    step = O.mean_angle_step(ang)
    ref = O.helical3d("BW", filtered, P.options.numpy(), ang, sp) * step
    assert rel_l2(rec, ref) < TOL
    # differentiable path: same numbers, gradient reaches the sinogram
    yt = torch.from_numpy(y).to(cuda).requires_grad_(True)
    rec2 = P.helical_fdk(yt, a)
    assert rel_l2(rec2.detach().cpu().numpy(), ref) < TOL
    rec2.square().sum().backward()
    assert yt.grad is not None and torch.isfinite(yt.grad).all() and float(yt.grad.abs().sum()) > 0


def test_helical_edge_cases(cuda):
    """One view, two views, no views, a batch of two, a square image."""
    P = _projector(image_size=(24, 24, 12))
    opts = P.options.numpy()
    for V in (1, 2):
        ang = _angles(V)
        sp = _source_pos(P, ang, True, seed=V)
        x, y = _inputs(P, V, seed=V)
        a, s = torch.from_numpy(ang).to(cuda), torch.from_numpy(sp).to(cuda)
        for op in OPS:
            inp = x if op in IMG_IN else y
            got = getattr(P, METHOD[op])(torch.from_numpy(inp).to(cuda), a, s).cpu().numpy()
            ref = O.helical3d(op, inp, opts, ang, sp)
            err = rel_l2(got, ref)
            assert err < TOL or (np.abs(ref).max() == 0 and np.abs(got).max() == 0), (V, op, err)
    ang0 = torch.zeros(0, device=cuda)
    out = P.backprojection_weighted(torch.zeros(1, 1, 0, 8, 64, device=cuda), ang0)
    assert out.shape == (1, 1, 12, 24, 24) and float(out.abs().sum()) == 0.0
    V = 120
    ang = _angles(V)
    sp = _source_pos(P, ang, False)
    x, y = _inputs(P, V, seed=2, batch=2)
    a, s = torch.from_numpy(ang).to(cuda), torch.from_numpy(sp).to(cuda)
    for op in ("A", "BW"):
        inp = x if op in IMG_IN else y
        got = getattr(P, METHOD[op])(torch.from_numpy(inp).to(cuda), a, s).cpu().numpy()
        assert rel_l2(got, O.helical3d(op, inp, opts, ang, sp)) < TOL, op


def test_helical_zero_offsets_equal_the_cone_arc_projector(cuda):
    """With source_pos = 0 the helical A equals Projector3d's cone-arc A, up
    to the cone-arc path's float32 boundary angles (the reference's circular
    CPU arithmetic; the helical operators take exact angles, as their
    fast-math CUDA reference is not float32-faithful): a few 1e-6."""
    from xrecon_b200 import Projector3d
    P = _projector()
    W, H, D = P.image_size
    C = Projector3d((W, H, D), P.num_det, P.pix_size, (3.0, 2.0), 300.0, 600.0, pixshift=(0.2, -0.3, 0.25),
                    binshift=(0.25, -0.1), scan_type="arc")
    V = 96
    ang = torch.from_numpy(_angles(V)).to(cuda)
    x, _ = _inputs(P, V, seed=6)
    xt = torch.from_numpy(x).to(cuda)
    sp = torch.zeros(4, V, device=cuda)
    hel = P.projection(xt, ang, sp)
    circ = C.projection(xt, ang)
    assert float((hel - circ).norm() / circ.norm()) < 1e-5
    assert math.isfinite(float(hel.sum()))
