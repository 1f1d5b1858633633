"""The Mayo direct-FDK route on the GPU: a synthetic DICOM-CT-PD series
loaded by xrecon_b200.mayo (pinned to the reference's loader on the CPU),
the helical projector it builds, and its filtered backprojection
(mayo_fdk.py:101-172 of the reference) against the FP64 helical oracle:
Bw(corr_u(sino * w, h)) * mean angle step * scale."""
import sys

import numpy as np
import pytest
import torch

from conftest import GOLDEN, rel_l2
from oracle import oracle as O

sys.path.insert(0, str(GOLDEN))
import mayo_series as MS  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["increasing", "decreasing"])
def test_mayo_direct_fdk_matches_oracle(cuda, tmp_path, case):
    from xrecon_b200 import mayo
    MS.write_series(tmp_path, case)
    cfg = mayo.MayoFdkConfig(data_dir=tmp_path, file_pattern="*.dcm", direct_fdk_scale=0.75,
                             **MS.CASES[case]["config"])
    prob = mayo.load_mayo_problem(cfg)
    P = mayo.make_helical_projector(prob.geometry, prob.sino.shape, prob.binshift, cuda, cfg)
    sino = torch.from_numpy(prob.sino).view(1, 1, *prob.sino.shape).to(cuda)
    ang = torch.from_numpy(prob.angles).to(cuda)
    sp = mayo.make_source_pos(prob.source_z, prob.shift_z, prob.shift_angle, prob.shift_radius, cuda)
    with torch.no_grad():
        rec = mayo.direct_fdk(P, sino, ang, sp, cfg).cpu().numpy()
    sw = prob.sino[None, None].astype(np.float64) * P.weight.cpu().numpy().astype(np.float64)
    filtered = O.correlate_rows(sw, P.filter.cpu().numpy().reshape(-1))
    ref = O.helical3d("BW", filtered, P.options.cpu().numpy(), prob.angles, sp.cpu().numpy())
    ref = ref * O.mean_angle_step(prob.angles) * cfg.direct_fdk_scale
    assert np.linalg.norm(ref) > 0
    assert rel_l2(rec, ref) < 1e-5
