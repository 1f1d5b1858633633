"""Fan/cone -> parallel rebinning on the GPU against the reference's own
rebin.py outputs (fixtures) and the FP64 oracle; the fused rebin + filter
pass against rebinning followed by the filter."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _kwargs(g, cuda):
    kw = {}
    for k in g:
        if k.startswith("kw_"):
            v = g[k]
            kw[k[3:]] = torch.from_numpy(v).to(cuda) if v.ndim else v.item()
    return kw


@pytest.mark.parametrize("case", ["arc4d", "flat5d", "arc5d_grid"])
def test_rebin_matches_reference_and_oracle(cuda, case):
    from xrecon_b200.rebin import fan_to_parallel_rebin
    g = load_golden(f"rebin_{case}")
    args = (float(g["iso_source"]), float(g["det_spacing"]), float(g["det_shift"]), str(g["detector_type"]))
    out, oa, t = fan_to_parallel_rebin(torch.from_numpy(g["sino"]).to(cuda), torch.from_numpy(g["angles"]).to(cuda),
                                       *args, **_kwargs(g, cuda))
    assert tuple(out.shape) == g["out"].shape
    assert rel_l2(t.cpu().numpy(), g["t"]) < 1e-6
    assert rel_l2(out.cpu().numpy(), g["out"]) < 1e-5
    kw_np = {k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in _kwargs(g, cuda).items()}
    exact, _, _ = O.fan_to_parallel_rebin(g["sino"], g["angles"], *args, **kw_np)
    assert rel_l2(out.cpu().numpy(), exact) < 1e-5


@pytest.mark.parametrize("case", ["arc4d", "flat5d"])
def test_fused_rebin_filter_matches_rebin_then_filter(cuda, case):
    from xrecon_b200.filters import filter_generate
    from xrecon_b200.rebin import fan_to_parallel_rebin
    g = load_golden(f"rebin_{case}")
    args = (float(g["iso_source"]), float(g["det_spacing"]), float(g["det_shift"]), str(g["detector_type"]))
    kw = _kwargs(g, cuda)
    sino = torch.from_numpy(g["sino"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    plain, _, t = fan_to_parallel_rebin(sino, ang, *args, **kw)
    Nt = plain.shape[-1]
    filt = filter_generate(Nt, float(t[1] - t[0]), "ramp", torch.float32).to(cuda)
    fused, _, _ = fan_to_parallel_rebin(sino, ang, *args, filt=filt, **kw)
    expect = O.correlate_rows(plain.cpu().numpy(), filt.cpu().numpy())
    assert rel_l2(fused.cpu().numpy(), expect) < 1e-5


def test_helical_rebin_matches_reference(cuda):
    from xrecon_b200.rebin import helical_cone_to_parallel_rebin
    g = load_golden("rebin_helical")
    out, oa, t, z = helical_cone_to_parallel_rebin(
        torch.from_numpy(g["sino"]).to(cuda), torch.from_numpy(g["angles"]).to(cuda),
        torch.from_numpy(g["source_z"]).to(cuda), 550.0, 0.005, 0.0, "arc",
        output_angles=torch.from_numpy(g["out_angles_in"]).to(cuda))
    assert rel_l2(out.cpu().numpy(), g["out"]) < 1e-5
    assert rel_l2(z.cpu().numpy(), g["out_source_z"]) < 1e-6
