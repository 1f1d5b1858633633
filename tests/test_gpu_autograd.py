"""Autograd Functions: backward = the hand-written transpose, checked against
the FP64 oracle's transpose (the reference's own autograd backward is the
partner transpose binding, xrecon/projector/functions.py:96-302), against
central finite differences, and the view-chunked least-squares Function on the
differentiable 3D cone-arc workload (B=8 x 128x128x32, 360 views, arc
detector 256x64)."""
import math

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _opts3d_arc(W, H, D, Nu, Nv, V=None):
    from xrecon_b200 import geometry as G
    geo = G.ConeBeam3d(G.Detector3d((Nu, Nv), (1.5, 1.5)), 500.0, 1000.0, "arc")
    return np.array(G.pack_options3d(G.Volume3d((W, H, D), 1.0), geo), np.float32)


PAIRS = [("Projection3d", "A", "AT"), ("ProjectionTranspose3d", "AT", "A"),
         ("BackProjection3d", "B", "BT"), ("BackProjectionTranspose3d", "BT", "B"),
         ("WeightedBackProjection3d", "BW", "BWT"), ("WeightedBackProjectionTranspose3d", "BWT", "BW")]


@pytest.mark.parametrize("name,op,adj", PAIRS)
def test_function_backward_is_oracle_transpose(cuda, name, op, adj):
    from xrecon_b200 import functions as F
    opts = _opts3d_arc(24, 20, 6, 40, 10)
    ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
    rng = np.random.default_rng(5)
    img_shape, sino_shape = (2, 1, 6, 20, 24), (2, 1, 30, 10, 40)
    x_shape, y_shape = (img_shape, sino_shape) if op in ("A", "BT", "BWT") else (sino_shape, img_shape)
    x = torch.from_numpy(rng.random(x_shape).astype(np.float32)).to(cuda).requires_grad_(True)
    up = rng.random(y_shape).astype(np.float32)
    out = getattr(F, name).apply(x, torch.from_numpy(opts).to(cuda), torch.from_numpy(ang).to(cuda))
    assert tuple(out.shape) == y_shape
    (g,) = torch.autograd.grad((out * torch.from_numpy(up).to(cuda)).sum(), x)
    exact = O.dd3d(adj, up, opts, ang)
    assert rel_l2(g.cpu().numpy(), exact) < 1e-5


FN2 = {"A": "Projection2d", "AT": "ProjectionTranspose2d", "B": "BackProjection2d", "BT": "BackProjectionTranspose2d",
       "BW": "WeightedBackProjection2d", "BWT": "WeightedBackProjectionTranspose2d"}


@pytest.mark.parametrize("scan", ["parallel", "flat", "arc"])
@pytest.mark.parametrize("dim", [2, 3])
def test_function_gradients_equal_the_reference_autograd_gradients(cuda, dim, scan):
    """The gradient each CUDA Function returns for the reference fixtures'
    input and upstream gradient equals the gradient the reference's own
    autograd Function returned (tests/golden/make_golden.py autograd, its
    CPU kernels behind functions.py:96-302), to 1e-5."""
    from conftest import load_golden
    from xrecon_b200 import functions as F
    g = load_golden(f"autograd{dim}d_{scan}")
    opts = torch.from_numpy(g["options"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    for op in ("A", "AT", "B", "BT", "BW", "BWT"):
        name = FN2[op] if dim == 2 else FN2[op][:-2] + "3d"
        x = torch.from_numpy(g[f"{op}_x"]).to(cuda).requires_grad_(True)
        out = getattr(F, name).apply(x, opts, ang)
        (grad,) = torch.autograd.grad((out * torch.from_numpy(g[f"{op}_u"]).to(cuda)).sum(), x)
        assert rel_l2(grad.cpu().numpy(), g[f"{op}_grad"]) < 1e-5, (dim, scan, op)


def _small_problem(cuda, B=2):
    opts = _opts3d_arc(32, 28, 8, 48, 12)
    ang = np.linspace(0, 2 * np.pi, 40, endpoint=False).astype(np.float32)
    rng = np.random.default_rng(11)
    x = rng.random((B, 1, 8, 28, 32)).astype(np.float32)
    y = rng.random((B, 1, 40, 12, 48)).astype(np.float32) * 10
    return opts, ang, x, y


def test_least_squares_gradient_matches_oracle(cuda):
    from xrecon_b200.functions import projection_least_squares
    opts, ang, x, y = _small_problem(cuda)
    xt = torch.from_numpy(x).to(cuda).requires_grad_(True)
    loss = projection_least_squares(xt, torch.from_numpy(y).to(cuda), torch.from_numpy(opts).to(cuda),
                                    torch.from_numpy(ang).to(cuda), view_chunk=7)
    (g,) = torch.autograd.grad(loss, xt)
    r = O.dd3d("A", x.astype(np.float64), opts, ang) - y
    assert abs(float(loss) - 0.5 * float(np.sum(r * r))) <= 1e-5 * 0.5 * float(np.sum(r * r))
    assert rel_l2(g.cpu().numpy(), O.dd3d("AT", r, opts, ang)) < 1e-5


def test_least_squares_chunking_is_exact(cuda):
    from xrecon_b200.functions import projection_least_squares
    opts, ang, x, y = _small_problem(cuda)
    res = []
    for chunk in (1, 7, 40):
        xt = torch.from_numpy(x).to(cuda).requires_grad_(True)
        loss = projection_least_squares(xt, torch.from_numpy(y).to(cuda), torch.from_numpy(opts).to(cuda),
                                        torch.from_numpy(ang).to(cuda), view_chunk=chunk)
        (g,) = torch.autograd.grad(loss, xt)
        res.append((float(loss), g.cpu().numpy()))
    for l, g in res[1:]:
        assert abs(l - res[0][0]) <= 1e-6 * abs(res[0][0])
        assert rel_l2(g, res[0][1]) < 1e-6


def test_least_squares_central_differences(cuda):
    """The loss is quadratic in x, so central differences are exact up to
    rounding; 64 random voxels."""
    from xrecon_b200.functions import projection_least_squares
    opts, ang, x, y = _small_problem(cuda, B=1)
    o, a, yt = torch.from_numpy(opts).to(cuda), torch.from_numpy(ang).to(cuda), torch.from_numpy(y).to(cuda)
    xt = torch.from_numpy(x).to(cuda).requires_grad_(True)
    (g,) = torch.autograd.grad(projection_least_squares(xt, yt, o, a, 16), xt)
    g = g.reshape(-1).cpu().numpy()
    rng = np.random.default_rng(3)
    idx = rng.choice(x.size, 64, replace=False)
    eps = 0.5
    fd = []
    for i in idx:
        xp = x.copy().reshape(-1); xp[i] += eps
        xm = x.copy().reshape(-1); xm[i] -= eps
        with torch.no_grad():
            lp = projection_least_squares(torch.from_numpy(xp.reshape(x.shape)).to(cuda), yt, o, a, 16)
            lm = projection_least_squares(torch.from_numpy(xm.reshape(x.shape)).to(cuda), yt, o, a, 16)
        fd.append((float(lp) - float(lm)) / (2 * eps))
    fd = np.array(fd)
    assert rel_l2(fd, g[idx]) < 1e-4


def _tv(x, eps=1e-6):
    dz = x[:, :, 1:, :-1, :-1] - x[:, :, :-1, :-1, :-1]
    dy = x[:, :, :-1, 1:, :-1] - x[:, :, :-1, :-1, :-1]
    dx = x[:, :, :-1, :-1, 1:] - x[:, :, :-1, :-1, :-1]
    return torch.sqrt(dx * dx + dy * dy + dz * dz + eps).sum()


def test_differentiable_cone_arc_workload(cuda):
    """B=8 volumes of 128x128x32 (1 mm), 360 views, arc detector 256x64 of
    1.5 mm, SOD 500 / SDD 1000.  Data: Poisson counts at 1e5 incident photons,
    log-transformed.  Loss ||Ax - y||^2 / 2 + 1e-3 TV(x) minimised by 50
    gradient steps through the chunked Function: the loss decreases
    monotonically, the adjoint test holds, and chunking keeps the peak memory
    of a gradient below one full sinogram."""
    from xrecon_b200 import backend as BK
    from xrecon_b200.functions import projection_least_squares
    from xrecon_b200.phantom import ellipsoid_volume_torch, random_ellipsoids3d
    opts = torch.from_numpy(_opts3d_arc(128, 128, 32, 256, 64)).to(cuda)
    ang = torch.linspace(0, 2 * math.pi, 361, device=cuda)[:-1].contiguous()
    torch.manual_seed(0)
    xs = [ellipsoid_volume_torch((32, 128, 128), random_ellipsoids3d(8, seed=100 + i, density=(0.0, 1.0)), cuda)
          for i in range(8)]
    x_true = (torch.stack(xs)[:, None] * 0.02).contiguous()  # attenuation in 1/mm
    p = BK.forward_projection3d(x_true, opts, ang)
    counts = torch.poisson(1e5 * torch.exp(-p)).clamp_min(1.0)
    y = -torch.log(counts / 1e5)
    # adjoint test on this geometry
    u = torch.rand_like(x_true)
    w = torch.rand_like(p)
    lhs = float((BK.forward_projection3d(u, opts, ang).double() * w.double()).sum())
    rhs = float((u.double() * BK.projection_transpose3d(w, opts, ang).double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    # step size from the operator norm (power iteration on A^T A)
    v = torch.rand_like(x_true)
    for _ in range(8):
        v = BK.projection_transpose3d(BK.forward_projection3d(v, opts, ang), opts, ang)
        lam = float(v.norm())
        v = v / lam
    step = 1.0 / lam
    x = torch.zeros_like(x_true, requires_grad=True)
    sino_bytes = p.numel() * p.element_size()
    losses = []
    for it in range(50):
        torch.cuda.reset_peak_memory_stats(cuda)
        base = torch.cuda.memory_allocated(cuda)
        ls = projection_least_squares(x, y, opts, ang, view_chunk=24)
        (g,) = torch.autograd.grad(ls, x)
        peak = torch.cuda.max_memory_allocated(cuda) - base
        assert peak < sino_bytes / 2, (peak, sino_bytes)
        tv = 1e-3 * _tv(x)
        (gt,) = torch.autograd.grad(tv, x)
        g = g + gt
        losses.append(float(ls) + float(tv))
        with torch.no_grad():
            x -= step * g
    assert all(b <= a * (1 + 1e-6) for a, b in zip(losses, losses[1:])), losses[:5]
    assert losses[-1] < 0.5 * losses[0]
