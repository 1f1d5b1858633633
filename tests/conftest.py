import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from xrecon_b200 import _native
    _native.lib()  # fail loudly if the extension is missing
    return torch.device("cuda:0")


@pytest.fixture(autouse=True)
def _oracle_tan_rounding(request):
    """GPU tests compare the CUDA path with the oracle in the CUDA path's own
    arithmetic: arc boundaries from tan rounded correctly to float32.  The
    reference's C library tanf differs from it by one unit for a few percent of
    arguments; the GPU tests check the reference fixtures separately."""
    if request.node.get_closest_marker("gpu") is None:
        yield
        return
    from oracle import oracle as O
    with O.tan_rounding(True):
        yield


@pytest.fixture(autouse=True)
def _device_error_word(request):
    """After every GPU test: no kernel may have reported a bounded-wait
    timeout through the device error word."""
    yield
    if request.node.get_closest_marker("gpu") is None:
        return
    import torch
    if not torch.cuda.is_available():
        return
    from xrecon_b200 import _native
    torch.cuda.synchronize()
    assert _native.device_error(clear=True) == 0, "a kernel reported a device error"
