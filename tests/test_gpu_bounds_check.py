"""The GPU parity suites again, on the bounds-checked build of the library.

libfcm_b200_debug.so is the same library compiled with -DFCM_BOUNDS_CHECK:
every grid point index, blob id from a tile or cell list, tile and cell id,
list slot, per-(blob, tile) partial, spectrum index of the fused x-transform and
Krylov column is checked (every kernel variant, through the autotuner's tests) against its range before the access; a kernel that
meets one outside counts it and skips the access (no trap).  This test runs the
parity suites in a child process with FCM_B200_BOUNDS_CHECK=1, where
tests/conftest.py requires every test to end with no violation
(fcm_debug_bounds), and the parity checks themselves must still pass, so the
checks change no result.  Nothing here makes an index go out of range on
purpose.
"""
import os
import subprocess
import sys

import pytest

from timstochrigidbodiessim_b200 import capi

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITES = ["tests/test_gpu_parity.py", "tests/test_gpu_config1_parity.py", "tests/test_gpu_tiles.py",
          "tests/test_gpu_shapes.py", "tests/test_gpu_batch.py", "tests/test_gpu_vs_reference.py",
          "tests/test_gpu_slip.py", "tests/test_gpu_dipoles.py", "tests/test_gpu_graph_step.py",
          "tests/test_gpu_autotune.py"]


def test_release_build_reports_unchecked(gpu):
    checked, count, site, index, limit = capi.debug_bounds()
    if os.environ.get("FCM_B200_BOUNDS_CHECK") == "1":
        assert checked
    else:
        assert not checked and count == 0 and site == "none"


def test_parity_suites_on_bounds_checked_build(gpu):
    if os.environ.get("FCM_B200_BOUNDS_CHECK") == "1":
        pytest.skip("already running on the bounds-checked build")
    assert os.path.exists(capi.DEBUG_LIB_PATH), "libfcm_b200_debug.so not built (python -m timstochrigidbodiessim_b200.build)"
    env = dict(os.environ, FCM_B200_BOUNDS_CHECK="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu", "-p", "no:cacheprovider"] + SUITES,
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    tail = (r.stdout + r.stderr)[-3000:]
    assert r.returncode == 0, tail
    assert " passed" in r.stdout and " failed" not in r.stdout, tail
