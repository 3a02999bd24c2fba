import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from fd3d_tsn_b200 import build
    build.build_oracle()
    if not os.path.exists(build.LIB):
        build.build_gpu()
    yield


@pytest.fixture(scope="session")
def gpu_available():
    from fd3d_tsn_b200 import solver
    return solver.device_count() > 0
