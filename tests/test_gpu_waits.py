"""Bounded device waits give up, report and return; the next call is correct.

The reference stops the process on a CUDA error (include/utils.h:7-11).  Here
every wait of a kernel on another agent is bounded: the projection kernel's
mbarrier waits for its TMA line windows and the ragged kernel's grid
barriers.  The failures are made on purpose without faulting anything: a test
hook makes the producer arm its barrier for a box but issue no copy (nothing
is in flight), or makes the grid barriers expect one block more than the
grid.  With short poll limits each wait runs out; the kernel sets its bit in
the device error word and returns.  The test checks the bit, that the launch
came back promptly, and that a normal call afterwards matches the oracle.
"""
import time

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def hooks_off():
    from xrecon_b200 import _native
    yield _native
    _native.test_hooks(0)
    _native.set_wait_limits(0, 0)
    torch.cuda.synchronize()
    _native.device_error(clear=True)


def test_tma_wait_times_out_and_next_call_is_correct(cuda, hooks_off):
    _native = hooks_off
    from xrecon_b200.backend import HostGeometry
    g = load_golden("dd3d_flat")
    geom = HostGeometry(3, g["options"].tolist()).struct
    assert _native.cell_plan(geom)["ok"], "the TMA path must be the one under test"
    x = torch.from_numpy(g["image"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    _native.apply(3, "A", x, geom, ang)  # warm: module loaded, plan cached
    torch.cuda.synchronize()
    assert _native.device_error(clear=True) == 0

    _native.set_wait_limits(256, 0)
    _native.test_hooks(1)
    t0 = time.perf_counter()
    _native.apply(3, "A", x, geom, ang)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    code = _native.device_error(clear=True)
    assert code & 1, f"no TMA timeout reported (error word {code:#x})"
    assert elapsed < 1.0, f"the stalled launch took {elapsed:.2f} s"
    with pytest.raises(RuntimeError, match="TMA transfer wait"):
        _native.set_wait_limits(256, 0)
        _native.apply(3, "A", x, geom, ang)
        _native.check_device_error()

    _native.test_hooks(0)
    _native.set_wait_limits(0, 0)
    _native.device_error(clear=True)
    got = _native.apply(3, "A", x, geom, ang).cpu().numpy()
    torch.cuda.synchronize()
    assert _native.device_error(clear=True) == 0
    assert rel_l2(got, O.dd3d("A", g["image"], g["options"], g["angles"])) < 1e-5


def test_ragged_barrier_times_out_and_next_launch_is_correct(cuda, hooks_off):
    _native = hooks_off
    from xrecon_b200 import geometry as G
    from xrecon_b200.phantom import create_phantom2d, random_ellipses2d
    from xrecon_b200.projector import Projector2d
    from xrecon_b200.ragged import RaggedFBP2d
    projectors = [Projector2d(G.Volume2d((48, 48), 1.0), G.FanBeam2d(G.Detector2d(72, 2.0), 500., 1000., "arc")),
                  Projector2d(G.Volume2d((40, 32), 1.0), G.FanBeam2d(G.Detector2d(64, 1.5), 400., 900., "flat"))]
    angles = [torch.from_numpy((np.arange(V) * (2 * np.pi / V)).astype(np.float32)) for V in (60, 45)]
    images = [torch.from_numpy(create_phantom2d((H, W), random_ellipses2d(5, seed=7 + i, n=max(W, H)))).to(cuda)
              for i, (H, W) in enumerate(((48, 48), (32, 40)))]
    R = RaggedFBP2d(projectors, angles, device=cuda)
    R(images)
    torch.cuda.synchronize()
    assert _native.device_error(clear=True) == 0

    _native.set_wait_limits(0, 1000)
    _native.test_hooks(2)
    t0 = time.perf_counter()
    R.launch()
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    code = _native.device_error(clear=True)
    assert code & 2, f"no barrier timeout reported (error word {code:#x})"
    assert elapsed < 1.0, f"the stalled launch took {elapsed:.2f} s"

    _native.test_hooks(0)
    _native.set_wait_limits(0, 0)
    _native.device_error(clear=True)
    sinos, recons = R(images)  # the barrier word and tile counters start from zero again
    torch.cuda.synchronize()
    assert _native.device_error(clear=True) == 0
    for P, a, im, s, r in zip(projectors, angles, images, sinos, recons):
        P = P.to(cuda)
        at = a.to(cuda)
        s_ref = P.projection(im[None, None], at)
        r_ref = P.filtered_backprojection(s_ref, at)
        assert rel_l2(s.cpu().numpy(), s_ref.cpu().numpy()) < 1e-6
        assert rel_l2(r.cpu().numpy(), r_ref.cpu().numpy()) < 1e-5
