"""The named 2D FBP and 3D FDK configurations at their full sizes on the GPU,
against the FP64 oracle (1e-5 relative L2).

* 2D fan-flat: a 256 x 256 image of 1 mm (Shepp-Logan plus 10 seeded
  ellipses), 720 views over 2 pi, 256 cells of 2 mm, SOD 500, SDD 1000: all
  six operators and the ramp FBP of the projection, whole.
* 3D cone-beam FDK geometry: 256 x 256 x 64 voxels of 1 mm (3D Shepp-Logan
  plus 20 seeded ellipsoids), 720 views, 384 x 96 cells of 1.5 mm, SOD 500,
  SDD 1000, flat and arc detectors.  The oracle cannot run the whole volume
  in a test, so it runs on crops that reproduce the GPU's arithmetic
  exactly: the voxel-owned outputs (B, Bw, A^T, FDK) on the central
  32 x 32 x 16 voxels (a volume geometry of exactly those voxels), the
  cell-owned ones (A, B^T, Bw^T) on the central 64 x 16 cells of every 8th
  view (a detector geometry of exactly those cells).  On the arc detector
  B^T and Bw^T walk each voxel's columns from its first one with chained
  angles, which a detector window cuts short, so they are checked on the
  flat detector only (the arc transposes are checked whole on smaller
  geometries in test_gpu_dd.py).
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_fan_flat_2d_fbp_configuration_whole(cuda):
    from xrecon_b200 import _native
    from xrecon_b200 import geometry as G
    from xrecon_b200.backend import HostGeometry
    from xrecon_b200.phantom import shepp_logan_plus_ellipses2d
    from xrecon_b200.projector import Projector2d
    P = Projector2d(G.Volume2d(256, 1.0), G.FanBeam2d(G.Detector2d(256, 2.0), 500.0, 1000.0, "flat")).to(cuda)
    opts = P.options.cpu().numpy()
    img = shepp_logan_plus_ellipses2d(256, 10, seed=1).astype(np.float32)[None, None]
    ang = (np.arange(720) * (2 * np.pi / 720)).astype(np.float32)
    at = torch.from_numpy(ang).to(cuda)
    x = torch.from_numpy(img).to(cuda)
    sino = P.projection(x, at)
    s_np = sino.cpu().numpy()
    assert rel_l2(s_np, O.dd2d("A", img, opts, ang)) < 1e-5
    recon = P.filtered_backprojection(sino, at).cpu().numpy()
    exact = O.filtered_backprojection2d(s_np, opts, ang, P.weight.cpu().numpy(), P.filter.cpu().numpy(),
                                        redundant=True, parker=None)
    assert rel_l2(recon, exact) < 1e-5
    geom = HostGeometry(2, opts.tolist()).struct
    rng = np.random.default_rng(12)
    y = rng.random(s_np.shape).astype(np.float32)
    for op, inp in (("AT", y), ("B", y), ("BW", y), ("BT", img), ("BWT", img)):
        got = _native.apply(2, op, torch.from_numpy(inp).to(cuda), geom, at).cpu().numpy()
        assert rel_l2(got, O.dd2d(op, inp, opts, ang)) < 1e-5, op


def _opts_c2(vol, det, scan):
    from xrecon_b200 import geometry as G
    geo = G.ConeBeam3d(G.Detector3d(det, (1.5, 1.5)), 500.0, 1000.0, scan)
    return np.array(G.pack_options3d(G.Volume3d(vol, 1.0), geo), np.float32)


@pytest.mark.parametrize("scan", ["flat", "arc"])
def test_cone_fdk_configuration_on_crops(cuda, scan):
    from xrecon_b200 import _native
    from xrecon_b200 import geometry as G
    from xrecon_b200.backend import HostGeometry
    from xrecon_b200.phantom import shepp_logan_plus_ellipsoids3d
    from xrecon_b200.projector import Projector3d
    P = Projector3d(G.Volume3d((256, 256, 64), 1.0),
                    G.ConeBeam3d(G.Detector3d((384, 96), (1.5, 1.5)), 500.0, 1000.0, scan)).to(cuda)
    opts = P.options.cpu().numpy()
    assert np.array_equal(opts, _opts_c2((256, 256, 64), (384, 96), scan))
    geom = HostGeometry(3, opts.tolist()).struct
    vol = shepp_logan_plus_ellipsoids3d((64, 256, 256), 20, seed=2).astype(np.float32)[None, None]
    ang = (np.arange(720) * (2 * np.pi / 720)).astype(np.float32)
    at = torch.from_numpy(ang).to(cuda)
    x = torch.from_numpy(vol).to(cuda)
    sino = _native.apply(3, "A", x, geom, at)
    s_np = sino.cpu().numpy()
    crop = (slice(None), slice(None), slice(24, 40), slice(112, 144), slice(112, 144))
    win = (slice(None), slice(None), slice(None, None, 8), slice(40, 56), slice(160, 224))
    opts_crop = _opts_c2((32, 32, 16), (384, 96), scan)
    opts_win = _opts_c2((256, 256, 64), (64, 16), scan)
    # cell-owned outputs on the detector window
    assert rel_l2(s_np[win], O.dd3d("A", vol, opts_win, ang[::8])) < 1e-5
    if scan == "flat":
        for op in ("BT", "BWT"):
            got = _native.apply(3, op, x, geom, at)[win].cpu().numpy()
            assert rel_l2(got, O.dd3d(op, vol, opts_win, ang[::8])) < 1e-5, op
    # voxel-owned outputs on the central crop, from the GPU's own sinogram
    for op in ("B", "BW", "AT"):
        got = _native.apply(3, op, sino, geom, at)[crop].cpu().numpy()
        assert rel_l2(got, O.dd3d(op, s_np, opts_crop, ang)) < 1e-5, op
    fdk = P.filtered_backprojection(sino, at)[crop].cpu().numpy()
    exact = O.filtered_backprojection3d(s_np, opts_crop, ang, P.weight.cpu().numpy(), P.filter.cpu().numpy())
    assert rel_l2(fdk, exact) < 1e-5
