import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def lib_built():
    from fastfusion_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def port_lib():
    from oracle import port
    port.build()
    return port
