import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "desert-search_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def dsg():
    """The product library, initialised on cuda:0."""
    import dsgpu
    dsgpu.init(0, 0.35)
    return dsgpu


@pytest.fixture(scope="session")
def ref_cpu():
    import libs
    r = libs.ref()
    if r is None:
        pytest.skip("reference pins (oracle/_ref) not built")
    return r
