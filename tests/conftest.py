import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Builds libcetagpu.so (if stale) and the CPU oracle once per session."""
    from cetasim_b200 import build
    build.build()
    build.build_oracle()
    return True


@pytest.fixture(scope="session")
def lib(built):
    from cetasim_b200 import _abi
    return _abi.load()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "faddeeva_golden.npz"))
