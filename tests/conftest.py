"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on the CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__ as entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


@pytest.fixture(scope="session")
def pkg():
    entry._load_build_module().build()
    return entry.load_package()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


@pytest.fixture(scope="session")
def gpu(pkg):
    n = pkg.device_count()
    if n < 1:
        raise RuntimeError("GPU test run without a CUDA device")
    return pkg


GOLDEN = os.path.join(ROOT, "tests", "golden")


def mask_dead(name, a, bc=0):
    """With the reference boundary passes, vm(imax, jmax+1) is written by bcUV from the previous
    content of the array (the top pass runs before the right-wall pass, boundary.f90:19-46) and
    is never read by the loop; it is excluded from comparisons."""
    if bc == 0 and (name.startswith("vm") or name == "vi"):
        a = a.copy()
        a[-1, -1] = 0.0
    return a


def fcopy(state):
    return {k: np.asfortranarray(v.copy()) for k, v in state.items()}
