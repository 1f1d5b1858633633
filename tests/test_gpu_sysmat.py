"""Sparse projection-matrix export on the GPU (Projector*.system_matrix)
against the reference's own matrices (fixtures from its system_matrix2d/3d
CPU code) and against the projection operator."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
# Entry-wise distance of the matrices.  Arc coefficients scale with the
# float32 boundary positions src.x + src.y tan(a), where the reference's C
# library tanf is one unit off for a few percent of angles (the CUDA path takes
# tan correctly rounded): those entries differ by up to 1e-4, which the
# operator comparisons below average out.
TOL = {"parallel": 1e-5, "flat": 1e-5, "arc": 5e-5}


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_system_matrix_matches_reference_and_projection(cuda, dim, scan):
    from xrecon_b200 import _native, backend as BK
    g = load_golden(f"sysmat{dim}d_{scan}")
    o = g["options"]
    geom = (_native.geom2d_from_values if dim == 2 else _native.geom3d_from_values)(o.tolist())
    M = _native.system_matrix(dim, geom, torch.from_numpy(g["angles"]), cuda)
    shape = tuple(int(s) for s in g["shape"])
    assert tuple(M.shape) == shape
    ref = np.zeros(shape)
    np.add.at(ref, (g["rows"], g["cols"]), g["vals"])
    got = M.to_dense().cpu().numpy().astype(np.float64)
    assert rel_l2(got, ref) < TOL[scan]
    # the matrix is the projection operator
    rng = np.random.default_rng(8)
    img_shape = (1, 1, int(o[1]), int(o[0])) if dim == 2 else (1, 1, int(o[2]), int(o[1]), int(o[0]))
    x = rng.random(img_shape).astype(np.float32)
    xt = torch.from_numpy(x).to(cuda)
    fwd = BK.forward_projection2d if dim == 2 else BK.forward_projection3d
    a = fwd(xt, torch.from_numpy(o).to(cuda), torch.from_numpy(g["angles"]).to(cuda)).reshape(-1)
    mx = torch.sparse.mm(M, xt.reshape(-1, 1)).reshape(-1)
    assert float((mx - a).norm() / a.norm()) < 1e-5
    exact = (O.dd2d if dim == 2 else O.dd3d)("A", x, o, g["angles"]).reshape(-1)
    assert rel_l2(mx.cpu().numpy(), exact) < 1e-5


def test_projector_system_matrix_follows_the_angles_device(cuda):
    """CPU angles give a CPU matrix (the reference builds and returns it on
    the CPU); CUDA angles give a CUDA matrix."""
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector2d
    P = Projector2d(G.Volume2d(16, 1.0), G.FanBeam2d(G.Detector2d(24, 2.0), 300.0, 600.0, "arc"))
    ang = torch.linspace(0, 3.0, 7)
    Mc = P.system_matrix(ang)
    assert not Mc.is_cuda and Mc.is_coalesced() and tuple(Mc.shape) == (7 * 24, 16 * 16)
    Mg = P.to(cuda).system_matrix(ang.to(cuda))
    assert Mg.is_cuda
    assert torch.equal(Mc.to_dense(), Mg.cpu().to_dense())
