"""The reference's own host code (its Projector2d / Projector3d, autograd
Functions and FBP pipeline, imported from the reference tree) driving this
package's backend module installed as ``xrecon_C`` (the one-line change of
INTEGRATION.md, Option 1).

There is no GPU here, so each backend function is wrapped: the wrapper
records the call and returns zeros of the output shape the options imply.
The test checks that every operator of the reference's classes, their
gradients and the FBP / FDK paths reach a function this module exports,
with the reference's own packed options, which must equal this package's
packing for the same geometry, and with the caller's angles.

Skipped where the reference tree is absent (it is found through
XRECON_REFERENCE_ROOT, or the root that oracle/build_oracle.py recorded when
it compiled the reference's CPU operators)."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]


def _reference_root():
    r = os.environ.get("XRECON_REFERENCE_ROOT")
    if not r:
        rec = ROOT / "oracle" / "_ref" / "reference_root.txt"
        r = rec.read_text().strip() if rec.exists() else ""
    if not r or not (Path(r) / "xrecon" / "projector" / "functions.py").is_file():
        pytest.skip("reference tree not available")
    return Path(r)


@pytest.fixture
def ref_with_backend(monkeypatch):
    root = _reference_root()
    monkeypatch.setattr(sys, "dont_write_bytecode", True)
    monkeypatch.syspath_prepend(str(root))
    from xrecon_b200 import backend
    calls = []

    def wrap(name):
        assert callable(getattr(backend, name))
        dim = 3 if name.endswith("3d") else 2

        def fake(inp, options, angles):
            o = options.detach().cpu().numpy().astype(np.float64)
            calls.append((name, o.copy(), angles.detach().cpu().numpy().copy()))
            lead = tuple(inp.shape[:2])
            V = int(angles.numel())
            sino_out = name.startswith(("forward_projection", "backward_projection_transpose",
                                        "weighted_backward_projection_transpose"))
            if dim == 3:
                W, H, D, Nu, Nv = (int(o[i]) for i in range(5))
                shape = lead + ((V, Nv, Nu) if sino_out else (D, H, W))
            else:
                W, H, Nu = int(o[0]), int(o[1]), int(o[2])
                shape = lead + ((V, Nu) if sino_out else (H, W))
            return torch.zeros(shape, dtype=inp.dtype)
        return fake

    names = [n for n in dir(backend) if n.endswith(("2d", "3d")) and not n.startswith("_")
             and "projection" in n]
    shim = type(sys)("xrecon_C")
    for n in names:
        setattr(shim, n, wrap(n))
    monkeypatch.setitem(sys.modules, "xrecon_C", shim)
    for m in [m for m in sys.modules if m == "xrecon" or m.startswith("xrecon.")]:
        monkeypatch.delitem(sys.modules, m)
    import xrecon
    import xrecon.projector.functions as RF
    RF._C = None
    return xrecon, calls


def test_reference_3d_projector_runs_on_this_backend(ref_with_backend):
    xrecon, calls = ref_with_backend
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector3d
    for scan in ("flat", "arc"):
        calls.clear()
        RP = xrecon.Projector3d(xrecon.Volume3d((20, 18, 6), (1.0, 1.1, 0.9), (0.2, -0.1, 0.3)),
                                xrecon.ConeBeam3d(xrecon.Detector3d((24, 8), (1.3, 1.2), (0.4, -0.2)),
                                                  500.0, 1000.0, scan))
        mine = Projector3d(G.Volume3d((20, 18, 6), (1.0, 1.1, 0.9), (0.2, -0.1, 0.3)),
                           G.ConeBeam3d(G.Detector3d((24, 8), (1.3, 1.2), (0.4, -0.2)), 500.0, 1000.0, scan))
        ang = torch.linspace(0.0, 6.0, 10)
        img = torch.rand(1, 1, 6, 18, 20, requires_grad=True)
        sino = torch.rand(1, 1, 10, 8, 24, requires_grad=True)
        RP.projection(img, ang).sum().backward()
        RP.backprojection(sino, ang).sum().backward()
        RP.backprojection_weighted(sino.detach(), ang)
        RP.projection_t(sino.detach(), ang)
        RP.backprojection_t(img.detach(), ang)
        RP.backprojection_weighted_t(img.detach(), ang)
        called = [c[0] for c in calls]
        assert called == ["forward_projection3d", "projection_transpose3d",
                          "backward_projection3d", "backward_projection_transpose3d",
                          "weighted_backward_projection3d", "projection_transpose3d",
                          "backward_projection_transpose3d", "weighted_backward_projection_transpose3d"], called
        n = len(calls)
        RP.filtered_backprojection(sino.detach(), ang)
        assert [c[0] for c in calls[n:]] == ["weighted_backward_projection3d"]
        for name, opts, a in calls:
            np.testing.assert_array_equal(opts.astype(np.float32), mine.options.numpy(), err_msg=name)
            np.testing.assert_array_equal(a, ang.numpy())


def test_reference_2d_projector_runs_on_this_backend(ref_with_backend):
    xrecon, calls = ref_with_backend
    from xrecon_b200 import geometry as G
    from xrecon_b200.projector import Projector2d
    for scan in ("parallel", "flat", "arc"):
        calls.clear()
        det = xrecon.Detector2d(30, 1.4, 0.3)
        geo = xrecon.ParallelBeam2d(det) if scan == "parallel" else xrecon.FanBeam2d(det, 400.0, 800.0, scan)
        RP = xrecon.Projector2d(xrecon.Volume2d((16, 14), (1.0, 1.2), (0.1, -0.2)), geo)
        mdet = G.Detector2d(30, 1.4, 0.3)
        mgeo = G.ParallelBeam2d(mdet) if scan == "parallel" else G.FanBeam2d(mdet, 400.0, 800.0, scan)
        mine = Projector2d(G.Volume2d((16, 14), (1.0, 1.2), (0.1, -0.2)), mgeo)
        ang = torch.linspace(0.0, 3.0, 12)
        img = torch.rand(2, 1, 14, 16, requires_grad=True)
        RP.projection(img, ang).sum().backward()
        sino = torch.rand(2, 1, 12, 30)
        RP.backprojection(sino, ang)
        RP.filtered_backprojection(sino, ang)
        called = [c[0] for c in calls]
        assert called[0] == "forward_projection2d" and called[1] == "projection_transpose2d", called
        assert called[2] in ("backward_projection2d", "back_projection2d"), called
        assert called[-1] in ("weighted_backward_projection2d", "weighted_back_projection2d"), called
        for name, opts, a in calls:
            np.testing.assert_array_equal(opts.astype(np.float32), mine.options.numpy(), err_msg=name)
