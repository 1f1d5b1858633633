"""The staged prefix backprojection (each view's row-prefix table footprint
copied into shared memory by TMA) against the unstaged gather and the oracle.

When every view is staged the arithmetic and its order are those of the
unstaged kernel, so the results are compared bit for bit.  The fallback
launch, which adds the views a CTA could not stage, is exercised with a test
hook that reports every odd view as not fitting (its views are then added
after the others: relative L2 1e-6 against the unstaged result, 1e-5 against
the oracle).  A stalled copy makes the staged kernel's bounded waits run out:
the error bit is set, the launch returns promptly and the next call is right.
"""
import time

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HOOK_TMA_STALL, HOOK_PFX_UNFIT, HOOK_PFX_NOSTAGE = 1, 4, 8


def _opts3d(W, H, D, Nu, Nv, dx, dy, dz, du, dv, sod, sdd, sh, shu, shv, scan):
    from xrecon_b200 import geometry as G
    det = G.Detector3d((Nu, Nv), (du, dv), (shu, shv))
    geo = G.ParallelBeam3d(det) if scan == "parallel" else G.ConeBeam3d(det, sod, sdd, scan)
    return np.array(G.pack_options3d(G.Volume3d((W, H, D), (dx, dy, dz), sh), geo), np.float32)


CASES = {
    "flat": [
        _opts3d(96, 80, 40, 128, 48, 1.0, 1.0, 1.0, 1.2, 1.2, 400., 800., (0.5, -0.3, 0.7), 0.3, -0.4, "flat"),
        _opts3d(64, 64, 24, 40, 12, 1.0, 1.0, 1.0, 2.5, 2.5, 300., 600., (4.0, -3.0, 2.0), 1.5, -1.0, "flat"),
        _opts3d(50, 70, 130, 96, 160, 1.0, 1.0, 1.0, 1.0, 1.0, 500., 900., 0.0, 0.0, 0.0, "flat"),
        _opts3d(40, 36, 200, 64, 300, 1.0, 1.0, 1.0, 1.3, 1.1, 450., 900., (0.2, 0.4, 60.0), -0.3, 20.0, "flat"),
    ],
    "arc": [
        _opts3d(96, 80, 40, 128, 48, 1.0, 1.0, 1.0, 1.2, 1.2, 400., 800., (0.5, -0.3, 0.7), 0.3, -0.4, "arc"),
        _opts3d(50, 70, 130, 96, 160, 1.0, 1.0, 1.0, 1.0, 1.0, 500., 900., 0.0, 0.0, 0.0, "arc"),
    ],
    "parallel": [
        _opts3d(96, 80, 40, 128, 48, 1.0, 1.0, 1.0, 1.2, 1.2, 400., 800., (0.5, -0.3, 0.7), 0.3, -0.4, "parallel"),
        _opts3d(50, 70, 130, 96, 160, 1.0, 1.0, 1.0, 1.0, 1.0, 500., 900., 0.0, 0.0, 0.0, "parallel"),
    ],
}


def _angles(n=24):
    ang = (np.arange(n) * (2 * np.pi / n) + 0.02).astype(np.float32)
    return np.concatenate([ang, np.array([np.pi / 4, 3 * np.pi / 4, -np.pi / 4], np.float32)])


@pytest.fixture
def native():
    from xrecon_b200 import _native
    _native.test_hooks(0)
    yield _native
    _native.test_hooks(0)
    _native.set_wait_limits(0, 0)
    torch.cuda.synchronize()
    _native.device_error(clear=True)


def _run(native, op, sino, opts, ang, dev, hooks):
    from xrecon_b200.backend import HostGeometry
    g = HostGeometry(3, np.asarray(opts).tolist()).struct
    native.test_hooks(hooks)
    y = native.apply(3, op, torch.from_numpy(sino).to(dev), g, torch.from_numpy(ang).to(dev))
    torch.cuda.synchronize()
    native.test_hooks(0)
    return y.cpu().numpy()


@pytest.mark.parametrize("scan", ["flat", "parallel", "arc"])
def test_staged_equals_unstaged_and_oracle(cuda, native, scan):
    from xrecon_b200.backend import HostGeometry
    ang = _angles()
    rng = np.random.default_rng(31)
    for opts in CASES[scan]:
        plan = native.pfx_stage_plan(HostGeometry(3, opts.tolist()).struct)
        assert plan["ok"], (scan, plan)
        sino = rng.random((1, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
        for op in ("B", "BW", "AT"):
            staged = _run(native, op, sino, opts, ang, cuda, 0)
            unstaged = _run(native, op, sino, opts, ang, cuda, HOOK_PFX_NOSTAGE)
            assert np.array_equal(staged, unstaged), (scan, op, float(np.abs(staged - unstaged).max()))
            assert rel_l2(staged, O.dd3d(op, sino, opts, ang)) < 1e-5, (scan, op)


@pytest.mark.parametrize("scan", ["flat", "parallel", "arc"])
def test_fallback_adds_the_views_not_staged(cuda, native, scan):
    ang = _angles()
    rng = np.random.default_rng(32)
    for opts in CASES[scan][:2]:
        sino = rng.random((2, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
        for op in ("B", "AT"):
            half = _run(native, op, sino, opts, ang, cuda, HOOK_PFX_UNFIT)
            unstaged = _run(native, op, sino, opts, ang, cuda, HOOK_PFX_NOSTAGE)
            assert rel_l2(half, unstaged) < 1e-6, (scan, op)
            assert rel_l2(half, O.dd3d(op, sino, opts, ang)) < 1e-5, (scan, op)
    assert native.device_error(clear=True) == 0


def test_staged_full_size_workload_subset(cuda, native):
    """The 512x512x256 / 1024x256 cone-flat geometry on 72 of its 1440 views,
    with the box the planner caps for it (its largest windows go to the
    fallback launch, which adds them after the others): staged B within
    1e-6 of unstaged B."""
    from xrecon_b200.backend import HostGeometry
    opts = np.asarray(load_golden("options")["c5_3d_flat"], np.float32)
    plan = native.pfx_stage_plan(HostGeometry(3, opts.tolist()).struct)
    assert plan["ok"], plan
    ang = (np.arange(0, 1440, 20) * (2 * np.pi / 1440)).astype(np.float32)
    sino = np.random.default_rng(33).random((1, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
    staged = _run(native, "B", sino, opts, ang, cuda, 0)
    unstaged = _run(native, "B", sino, opts, ang, cuda, HOOK_PFX_NOSTAGE)
    assert rel_l2(staged, unstaged) < 1e-6, rel_l2(staged, unstaged)


def test_staged_wait_times_out_and_next_call_is_correct(cuda, native):
    opts = CASES["flat"][0]
    ang = _angles()
    sino = np.random.default_rng(34).random((1, 1, ang.size, int(opts[4]), int(opts[3]))).astype(np.float32)
    _run(native, "B", sino, opts, ang, cuda, 0)  # warm: module loaded, plans cached
    assert native.device_error(clear=True) == 0
    native.set_wait_limits(256, 0)
    t0 = time.perf_counter()
    _run(native, "B", sino, opts, ang, cuda, HOOK_TMA_STALL)
    elapsed = time.perf_counter() - t0
    code = native.device_error(clear=True)
    assert code & 1, f"no TMA timeout reported (error word {code:#x})"
    assert elapsed < 1.0, f"the stalled launch took {elapsed:.2f} s"
    native.set_wait_limits(0, 0)
    got = _run(native, "B", sino, opts, ang, cuda, 0)
    assert native.device_error(clear=True) == 0
    assert rel_l2(got, O.dd3d("B", sino, opts, ang)) < 1e-5


@pytest.mark.parametrize("case", ["ffs", "reverse", "half_scan"])
def test_helical_staged_equals_unstaged(cuda, native, case):
    """Helical B and A^T (per-view z placement and column pitch, views whose
    z reach misses a run skipped): staged equals unstaged bit for bit; with
    every odd view left to the fallback, within 1e-6."""
    from test_gpu_helical import CASES as HCASES, METHOD, _case_angles, _inputs, _projector, _source_pos
    over, ffs = HCASES[case]
    P = _projector(**over)
    V = 240
    ang = _case_angles(case, V)
    sp = _source_pos(P, ang, ffs)
    _, y = _inputs(P, V, batch=2)
    a, s, yt = torch.from_numpy(ang).to(cuda), torch.from_numpy(sp).to(cuda), torch.from_numpy(y).to(cuda)

    def run(op, hooks):
        native.test_hooks(hooks)
        out = getattr(P, METHOD[op])(yt, a, s)
        torch.cuda.synchronize()
        native.test_hooks(0)
        return out.cpu().numpy()

    for op in ("B", "AT"):
        staged, unstaged = run(op, 0), run(op, HOOK_PFX_NOSTAGE)
        assert np.array_equal(staged, unstaged), (case, op, float(np.abs(staged - unstaged).max()))
        assert rel_l2(run(op, HOOK_PFX_UNFIT), unstaged) < 1e-6, (case, op)
        assert rel_l2(staged, O.helical3d(op, y, P.options.numpy(), ang, sp)) < 1e-5, (case, op)
    assert native.device_error(clear=True) == 0
