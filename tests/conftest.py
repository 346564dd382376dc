import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def orc():
    from tests import oracle_lib

    return oracle_lib.load()


@pytest.fixture(scope="session")
def gpu():
    import phiray_b200 as px

    g = px.Gpu(0)
    yield g
    g.close()
