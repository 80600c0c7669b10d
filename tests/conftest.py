import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cb():
    """The product package; the library must have been built (python cfd_b200/build.py)."""
    import cfd_b200
    return cfd_b200


@pytest.fixture(scope="session")
def gpu(cb):
    if not cb.device_available():
        pytest.skip("no CUDA device")
    return cb
