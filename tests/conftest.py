import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and runs the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from meshfemsparse_b200.build import build_library
    from oracle.build import build_oracle
    build_library()
    build_oracle()
    yield
