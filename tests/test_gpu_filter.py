"""The FBP row filter (xr_fbp_filter): the FFT kernel against an FP64 direct
correlation, and against the direct-sum kernel the plain switch selects.

The filter is out[i] = sum_j x[j] filt[j - i + Nu - 1] (the reference's
conv2d / conv3d with padding Nu - 1, projector.py:201, projector3d.py:190).
The FFT kernel handles Nu <= 2048 (transform length <= 4096); wider rows take
the direct kernel.  Tolerance: 2e-6 relative L2 on random rows with random
filters, 2e-5 on projection-like rows with the ramp filter, whose output
cancels much of its input (the FP32 direct sum is at 1e-6 there).
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _corr64(x, f):
    Nu = x.shape[-1]
    W = np.lib.stride_tricks.sliding_window_view(f.astype(np.float64), Nu)[::-1]  # W[i] = f[Nu-1-i : 2Nu-1-i]
    return x.reshape(-1, Nu).astype(np.float64) @ W.T


def _ramp(Nu, d):
    x = np.arange(2 * Nu - 1) - Nu + 1
    h = np.zeros(2 * Nu - 1)
    odd = x % 2 != 0
    h[odd] = -1.0 / (np.pi ** 2 * d ** 2 * x[odd] ** 2)
    h[Nu - 1] = 1.0 / (4 * d ** 2)
    return h.astype(np.float32)


@pytest.fixture
def plain_off():
    from xrecon_b200 import _native
    yield _native
    _native.set_plain_kernels(0)


@pytest.mark.parametrize("Nu,nrows", [(1, 3), (2, 1), (3, 5), (7, 2), (64, 9), (100, 33), (257, 16),
                                      (736, 17), (1024, 64), (2048, 5), (2049, 3)])
def test_filter_random_rows_and_taps(cuda, plain_off, Nu, nrows):
    _native = plain_off
    rng = np.random.default_rng(Nu * 7 + nrows)
    x = rng.standard_normal((nrows, Nu)).astype(np.float32)
    f = rng.standard_normal(2 * Nu - 1).astype(np.float32)
    xt, ft = torch.from_numpy(x).to(cuda), torch.from_numpy(f).to(cuda)
    got = _native.fbp_filter(xt, nview=nrows, rows_per_view=1, cosw=None, filt=ft, parker=None).cpu().numpy()
    ref = _corr64(x, f)
    assert rel_l2(got.reshape(ref.shape), ref) < 2e-6
    _native.set_plain_kernels(1)
    direct = _native.fbp_filter(xt, nview=nrows, rows_per_view=1, cosw=None, filt=ft, parker=None).cpu().numpy()
    assert rel_l2(direct.reshape(ref.shape), ref) < 2e-6


@pytest.mark.parametrize("Nu", [256, 384, 1024])
def test_filter_ramp_on_projections_with_weights(cuda, plain_off, Nu):
    _native = plain_off
    rng = np.random.default_rng(Nu)
    t = np.linspace(-1.0, 1.0, Nu)
    nv, nr = 12, 3
    rows = []
    for _ in range(nv * nr):
        c, w = rng.uniform(-0.5, 0.5), rng.uniform(0.2, 0.9)
        r = np.sqrt(np.clip(1 - ((t - c) / w) ** 2, 0, None)) * rng.uniform(50, 300)
        r += np.sqrt(np.clip(1 - ((t - 0.5 * c) / (0.3 * w)) ** 2, 0, None)) * rng.uniform(0, 30)
        rows.append(r)
    x = np.array(rows, np.float32).reshape(nv, nr, Nu)
    cosw = (np.cos(np.linspace(-0.4, 0.4, Nu))).astype(np.float32)
    parker = rng.uniform(0.0, 1.0, (nv, Nu)).astype(np.float32)
    f = _ramp(Nu, 0.55)
    got = _native.fbp_filter(torch.from_numpy(x).to(cuda), nview=nv, rows_per_view=nr,
                             cosw=torch.from_numpy(cosw), filt=torch.from_numpy(f),
                             parker=torch.from_numpy(parker)).cpu().numpy()
    xw = x.astype(np.float64) * cosw[None, None, :] * parker[:, None, :]
    ref = _corr64(xw.astype(np.float32), f).reshape(x.shape)
    assert rel_l2(got, ref) < 2e-5


def test_filter_half_precision_input(cuda):
    from xrecon_b200 import _native
    rng = np.random.default_rng(5)
    Nu = 300
    x = rng.standard_normal((10, Nu)).astype(np.float32)
    f = rng.standard_normal(2 * Nu - 1).astype(np.float32)
    for dt in (torch.float16, torch.bfloat16):
        xt = torch.from_numpy(x).to(cuda).to(dt)
        got = _native.fbp_filter(xt, nview=10, rows_per_view=1, cosw=None, filt=torch.from_numpy(f),
                                 parker=None).cpu().numpy()
        ref = _corr64(xt.float().cpu().numpy(), f)
        assert rel_l2(got, ref) < 2e-6
