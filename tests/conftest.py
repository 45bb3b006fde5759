import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """The GPU library, loaded.  A GPU test fails (it is not skipped) when a GPU
    driver is present but CUDA is unusable; it is skipped only on machines
    without any NVIDIA driver."""
    if not _cuda_available():
        if shutil.which("nvidia-smi") is None:
            pytest.skip("no GPU on this machine")
        pytest.fail("nvidia-smi exists but CUDA is unavailable")
    from timstochrigidbodiessim_b200 import capi
    return capi.load()


@pytest.fixture(autouse=True)
def _bounds_checked_run():
    """With FCM_B200_BOUNDS_CHECK=1 the bounds-checked library is loaded
    (timstochrigidbodiessim_b200.capi); then every test that touched the GPU must
    end with no device index outside its range (fcm_debug_bounds)."""
    if os.environ.get("FCM_B200_BOUNDS_CHECK") != "1" or not _cuda_available():
        yield
        return
    from timstochrigidbodiessim_b200 import capi
    capi.debug_bounds(reset=True)
    yield
    checked, count, site, index, limit = capi.debug_bounds(reset=True)
    assert checked, "FCM_B200_BOUNDS_CHECK=1 but the release library is loaded"
    assert count == 0, "%d device indices out of range; first: %s %d of %d" % (count, site, index, limit)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
