"""Ragged batches in one persistent launch (xr_ragged2d_run) against the
per-instance operators (each already pinned to the oracle) and, for small
instances, the FP64 oracle itself."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _mixed_batch():
    from xrecon_b200 import geometry as G
    from xrecon_b200.phantom import create_phantom2d, random_ellipses2d
    from xrecon_b200.projector import Projector2d
    specs = [((64, 64), 1.0, G.FanBeam2d(G.Detector2d(96, 2.0), 500., 1000., "arc"), 90),
             ((48, 40), (1.0, 1.2), G.FanBeam2d(G.Detector2d(80, 1.5, 0.3), 400., 900., "flat"), 72),
             ((32, 32), 1.0, G.ParallelBeam2d(G.Detector2d(50, 1.0)), 60),
             ((80, 80), 0.8, G.FanBeam2d(G.Detector2d(128, 1.2, -0.6), 450., 800., "arc"), 120),
             ((100, 100), 0.5, G.FanBeam2d(G.Detector2d(150, 1.0), 600., 1200., "flat"), 200)]
    projectors, angles, images = [], [], []
    for i, (size, pix, geo, V) in enumerate(specs):
        projectors.append(Projector2d(G.Volume2d(size, pix), geo))
        angles.append((np.arange(V) * (2 * np.pi / V) + 0.01 * i).astype(np.float32))
        W, H = size
        images.append(create_phantom2d((H, W), random_ellipses2d(6, seed=40 + i, n=max(W, H))))
    return projectors, angles, images


def _per_instance(projectors, angles, images, cuda):
    out = []
    for P, a, im in zip(projectors, angles, images):
        P = P.to(cuda)
        at = torch.from_numpy(a).to(cuda)
        x = torch.from_numpy(im)[None, None].to(cuda)
        s = P.projection(x, at)
        out.append((s.cpu().numpy(), P.filtered_backprojection(s, at).cpu().numpy()))
    return out


def test_ragged_matches_per_instance_and_oracle(cuda):
    from xrecon_b200.ragged import RaggedFBP2d
    projectors, angles, images = _mixed_batch()
    R = RaggedFBP2d(projectors, [torch.from_numpy(a) for a in angles], device=cuda)
    sinos, recons = R([torch.from_numpy(im).to(cuda) for im in images])
    ref = _per_instance(projectors, angles, images, cuda)
    for i, ((s_ref, r_ref), s, r) in enumerate(zip(ref, sinos, recons)):
        assert rel_l2(s.cpu().numpy(), s_ref) < 1e-6, i
        assert rel_l2(r.cpu().numpy(), r_ref) < 1e-5, i
    for i in (0, 3):  # the FP64 oracle on two instances
        P = projectors[i]
        opts = P.options.cpu().numpy()
        s_ex = O.dd2d("A", images[i][None, None], opts, angles[i])
        r_ex = O.filtered_backprojection2d(s_ex, opts, angles[i], P.weight.cpu().numpy(), P.filter.cpu().numpy(),
                                           redundant=True, parker=None)
        assert rel_l2(sinos[i].cpu().numpy(), s_ex) < 1e-5
        assert rel_l2(recons[i].cpu().numpy(), r_ex) < 1e-5


def test_ragged_tile_configs_and_graph_replay_agree(cuda):
    from xrecon_b200.ragged import RaggedFBP2d
    projectors, angles, images = _mixed_batch()
    R = RaggedFBP2d(projectors, [torch.from_numpy(a) for a in angles], device=cuda, autotune=False, graph=False)
    R.set_images([torch.from_numpy(im).to(cuda) for im in images])
    base = None
    for a in range(4):
        for v in range(4):
            R.launch(True, (a, v))
            torch.cuda.synchronize()
            got = (R.sino.clone(), R.recon.clone())
            if base is None:
                base = got
            else:
                assert float((got[0] - base[0]).norm() / base[0].norm()) < 1e-6, (a, v)
                assert float((got[1] - base[1]).norm() / base[1].norm()) < 1e-5, (a, v)
    R.capture()
    R.recon.zero_()
    R.run()
    torch.cuda.synchronize()
    assert float((R.recon - base[1]).norm() / base[1].norm()) < 1e-5
    # new images through the same graph
    R.set_images([torch.from_numpy(2.0 * im).to(cuda) for im in images])
    R.run()
    torch.cuda.synchronize()
    assert float((R.recon - 2.0 * base[1]).norm() / (2.0 * base[1]).norm()) < 1e-5


def test_ragged_fan_arc_workload_64_instances(cuda):
    """The 64-instance fan-arc batch (seed 4): every instance agrees with its
    per-instance projection and FBP (two FP32 summation orders: the FBP sums
    up to 1440 views of mixed-sign filtered values), and the cheapest
    instances match the FP64 oracle; one autotuned graph replay."""
    sys.path.insert(0, str(ROOT))
    import bench
    from xrecon_b200.ragged import RaggedFBP2d
    projectors, angles, images = bench.ragged_c4_batch()
    R = RaggedFBP2d(projectors, [torch.from_numpy(a) for a in angles], device=cuda)
    sinos, recons = R([torch.from_numpy(im).to(cuda) for im in images])
    torch.cuda.synchronize()
    ref = _per_instance(projectors, angles, images, cuda)
    worst = (0.0, 0.0)
    for i, ((s_ref, r_ref), s, r) in enumerate(zip(ref, sinos, recons)):
        es, er = rel_l2(s.cpu().numpy(), s_ref), rel_l2(r.cpu().numpy(), r_ref)
        worst = (max(worst[0], es), max(worst[1], er))
    print(f"\nragged vs per-instance: sinogram {worst[0]:.2e}, reconstruction {worst[1]:.2e}")
    assert worst[0] < 1e-6 and worst[1] < 5e-5
    cost = [P.image_size[0] ** 2 * a.size for P, a in zip(projectors, angles)]
    for i in np.argsort(cost)[:3]:
        P = projectors[i]
        opts = P.options.cpu().numpy()
        s_ex = O.dd2d("A", images[i][None, None], opts, angles[i])
        r_ex = O.filtered_backprojection2d(s_ex, opts, angles[i], P.weight.cpu().numpy(), P.filter.cpu().numpy(),
                                           redundant=True, parker=None)
        es, er = rel_l2(sinos[i].cpu().numpy(), s_ex), rel_l2(recons[i].cpu().numpy(), r_ex)
        ep = rel_l2(ref[i][1], r_ex)
        print(f"instance {i}: vs oracle sinogram {es:.2e}, reconstruction {er:.2e} (per-instance path {ep:.2e})")
        assert es < 1e-5 and er < 1e-5
    info = R.info()
    assert info["grid"] >= 148
