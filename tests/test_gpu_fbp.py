"""FBP / FDK on the GPU through Projector2d/3d.filtered_backprojection, against
the FP64 oracle (1e-5) and the reference's own reconstructions (1e-5, arc
included).  The geometries are those of tests/golden/make_golden.py, rebuilt
with this package's geometry classes."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES2D = {
    "flat_ramp": ("flat", "ramp", False),
    "arc_ramp": ("arc", "ramp", False),
    "parallel_shepplogan": ("parallel", "shepplogan", False),
    "flat_hann": ("flat", "hann", False),
    "flat_parker": ("flat", "ramp", True),
}


def _projector2d(scan, filt):
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector2d
    if scan == "parallel":
        geo = G.ParallelBeam2d(G.Detector2d(96, 1.0))
    else:
        geo = G.FanBeam2d(G.Detector2d(96, 2.0), 500.0, 1000.0, scan)
    return Projector2d(G.Volume2d(64, 1.0), geo, filter_type=filt)


def _projector3d(scan):
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector3d
    geo = G.ConeBeam3d(G.Detector3d((48, 12), (1.5, 1.5)), 500.0, 1000.0, scan)
    return Projector3d(G.Volume3d((32, 32, 8), 1.0), geo)


@pytest.mark.parametrize("case", sorted(CASES2D))
def test_fbp2d_matches_oracle_and_reference(cuda, case):
    scan, filt, parker = CASES2D[case]
    g = load_golden(f"fbp2d_{case}")
    P = _projector2d(scan, filt).to(cuda)
    np.testing.assert_allclose(P.options.cpu().numpy(), g["options"], rtol=0, atol=0)
    sino = torch.from_numpy(g["sino"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    recon = P.filtered_backprojection(sino, ang, parker=parker).cpu().numpy()
    pk = g["parker"].reshape(1, 1, g["angles"].size, -1) if parker else None
    exact = O.filtered_backprojection2d(g["sino"], g["options"], g["angles"], P.weight.cpu().numpy(),
                                        P.filter.cpu().numpy(), redundant=not parker, parker=pk)
    assert rel_l2(recon, exact) < 1e-5
    assert rel_l2(recon, g["recon"]) < 1e-5


@pytest.mark.parametrize("scan", ["flat", "arc"])
def test_fdk3d_matches_oracle_and_reference(cuda, scan):
    g = load_golden(f"fdk3d_{scan}")
    P = _projector3d(scan).to(cuda)
    np.testing.assert_allclose(P.options.cpu().numpy(), g["options"], rtol=0, atol=0)
    sino = torch.from_numpy(g["sino"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    recon = P.filtered_backprojection(sino, ang).cpu().numpy()
    exact = O.filtered_backprojection3d(g["sino"], g["options"], g["angles"], P.weight.cpu().numpy(),
                                        P.filter.cpu().numpy())
    assert rel_l2(recon, exact) < 1e-5
    assert rel_l2(recon, g["recon"]) < 1e-5


@pytest.mark.parametrize("scan", ["flat", "arc"])
def test_fdk3d_differentiable_path_matches_fused_path(cuda, scan):
    """With gradients required the FDK runs torch weighting/filtering and the
    weighted-backprojection Function; it must give the fused result and a
    gradient equal to the adjoint chain applied to the upstream gradient."""
    g = load_golden(f"fdk3d_{scan}")
    P = _projector3d(scan).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    fused = P.filtered_backprojection(torch.from_numpy(g["sino"]).to(cuda), ang)
    sino = torch.from_numpy(g["sino"]).to(cuda).requires_grad_(True)
    recon = P.filtered_backprojection(sino, ang)
    assert rel_l2(recon.detach().cpu().numpy(), fused.cpu().numpy()) < 1e-5
    gen = torch.Generator(device=cuda).manual_seed(11)
    up = torch.randn(recon.shape, device=cuda, generator=gen)
    (grad,) = torch.autograd.grad((recon * up).sum(), sino)
    # <FDK(d), up> = <d, FDK^T(up)>: check against a directional derivative.
    # The sums cancel to a small fraction of their terms, so the bound is
    # taken relative to the norms (Cauchy-Schwarz), not to the sums.  On the
    # arc detector B / Bw take the chain's linear step and their transposes
    # the exact one, so the pair is adjoint to ~1e-6 of the norms, not to
    # rounding.
    d = torch.randn(sino.shape, device=cuda, generator=gen)
    fd = P.filtered_backprojection(d, ang).double()
    lhs = float((grad.double() * d.double()).sum())
    rhs = float((fd * up.double()).sum())
    scale = float(fd.norm() * up.double().norm())
    assert abs(lhs - rhs) <= 1e-5 * scale


def test_fbp2d_trainable_filter_and_weight_gradients(cuda):
    """Gradients of the FBP with respect to a trainable filter and cosine
    weight against torch autograd of the same pipeline in FP64 on the CPU
    (weights x correlation through conv2d, then the oracle's Bw)."""
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector2d
    g = load_golden("fbp2d_flat_ramp")
    geo = G.FanBeam2d(G.Detector2d(96, 2.0), 500.0, 1000.0, "flat")
    P = Projector2d(G.Volume2d(64, 1.0), geo, filter_type="ramp", trainable=True).to(cuda)
    sino = torch.from_numpy(g["sino"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    up = np.random.default_rng(2).random((1, 1, 64, 64))
    recon = P.filtered_backprojection(sino, ang)
    (recon * torch.from_numpy(up).float().to(cuda)).sum().backward()
    # FP64 CPU reference: d/dfilt and d/dweight of <FBP(sino), up>
    Nu = 96
    w = P.weight.detach().cpu().double().requires_grad_(True)
    f = P.filter.detach().cpu().double().requires_grad_(True)
    s = torch.from_numpy(g["sino"]).double()
    filtered = torch.nn.functional.conv2d(s * w, f.reshape(1, 1, 1, -1), padding=(0, Nu - 1))
    # the weighted backprojection is linear: contract with Bw^T(up) instead
    bwt = torch.from_numpy(O.dd2d("BWT", up, g["options"], g["angles"]))
    scale = float(O.mean_angle_step(g["angles"])) / 2
    (filtered * bwt * scale).sum().backward()
    assert rel_l2(P.filter.grad.cpu().numpy(), f.grad.numpy()) < 1e-5
    assert rel_l2(P.weight.grad.cpu().numpy(), w.grad.numpy()) < 1e-5
