import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "virial-engine_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the CUDA library)")
    config.addinivalue_line("markers", "slow: long physical check")


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def vl():
    """The CUDA library's Python mirror (loads libvirial_lj.so)."""
    import virial_lj
    return virial_lj


@pytest.fixture(scope="session")
def gpu(vl):
    if vl.device_count() == 0:
        pytest.fail("no CUDA device visible: GPU tests need one")
    return vl
