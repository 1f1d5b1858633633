"""xr_dd2d_noalloc: the 2D entry point for callers that cannot allocate
device memory while they run (a service with a device-memory budget fixed at
start-up, or code inside a host framework that owns the device allocator).
Its scratch is a fixed static device array inside the library.  Called
through the C ABI and compared with xr_dd2d (caller workspace) on
consecutive calls.  Named to be collected last, so that it also runs after
every other test has used the library.
"""
import ctypes
import math

import pytest
import torch

from xrecon_b200 import _native

pytestmark = pytest.mark.gpu

XR_ERR_WORKSPACE = 2
SCRATCH_BYTES = 32 << 20


def _geom(scan_type):
    # 2D fan geometry (effective detector spacing as the packed options).
    return _native.Geom2d(W=96, H=80, Nu=160, type=scan_type, dx=1.0, dy=1.0,
                          du=1.1 if scan_type != 2 else 0.0016, sod=500.0, sdd=900.0,
                          shift_x=0.7, shift_y=-1.3, shift_u=0.4 if scan_type != 2 else 0.0005)


def _noalloc(op, x, geom, ang, out):
    L = _native.lib()
    rc = L.xr_dd2d_noalloc(_native.OPS[op], ctypes.byref(geom), x.data_ptr(), _native.DTYPES[x.dtype],
                           out.data_ptr(), _native.DTYPES[out.dtype], ang.data_ptr(), x.shape[0] * x.shape[1],
                           ang.numel(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.xr_last_error().decode()
    return out


@pytest.mark.parametrize("scan_type", [0, 1, 2])
def test_noalloc_matches_workspace_entry_on_consecutive_calls(cuda, scan_type):
    g = torch.Generator(device="cpu").manual_seed(11 + scan_type)
    geom = _geom(scan_type)
    V = 120
    ang = torch.linspace(0.0, 2.0 * math.pi, V + 1)[:-1].add(0.01).to(cuda)
    img = torch.rand(2, 1, geom.H, geom.W, generator=g).to(cuda)
    sino = torch.rand(2, 1, V, geom.Nu, generator=g).to(cuda)
    # two rounds of consecutive calls over every operator: each call reuses
    # the same static scratch left behind by a different operator
    for _ in range(2):
        for op in ("A", "BT", "BWT", "AT", "B", "BW"):
            x = img if op in _native.SINO_OUT else sino
            want = _native.apply(2, op, x, geom, ang)
            got = _noalloc(op, x, geom, ang, torch.full_like(want, float("nan")))
            torch.cuda.synchronize()
            assert torch.equal(got, want), f"{op}: max diff {(got - want).abs().max().item()}"


def test_noalloc_rejects_oversized_requests(cuda):
    geom = _geom(1)
    ang = torch.zeros(12000, device=cuda)
    need = _native.lib().xr_dd2d_workspace_size(0, ctypes.byref(geom), 1, ang.numel())
    assert need > SCRATCH_BYTES
    img = torch.ones(1, 1, geom.H, geom.W, device=cuda)
    out = torch.zeros(1, 1, ang.numel(), geom.Nu, device=cuda)
    L = _native.lib()
    rc = L.xr_dd2d_noalloc(0, ctypes.byref(geom), img.data_ptr(), 0, out.data_ptr(), 0, ang.data_ptr(), 1,
                           ang.numel(), torch.cuda.current_stream().cuda_stream)
    assert rc == XR_ERR_WORKSPACE
    assert "fixed" in L.xr_last_error().decode()
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0
