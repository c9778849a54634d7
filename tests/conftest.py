import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the native CUDA path")


@pytest.fixture(scope="session", autouse=True)
def _native_built():
    """Build the checker (oracle) and the product library once per session."""
    from oracle import oracle
    oracle.build()
    from falconnpp_b200 import _build
    _build.build()
    yield
