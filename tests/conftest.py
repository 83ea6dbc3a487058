import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a path")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native library and the oracle once per session (no-op when fresh)."""
    from ma57_b200 import build as nb
    nb.build()
    from oracle import pyoracle
    pyoracle.build()
    yield
