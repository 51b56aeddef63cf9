import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and the CUDA library in-tree (no-ops when up to date)."""
    from oracle import pyoracle
    if not os.path.exists(pyoracle.LIB_PATH):
        pyoracle.build()
    from lbm_b200 import build
    build.build()
    yield
