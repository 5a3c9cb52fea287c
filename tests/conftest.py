import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a engine)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def engine():
    """The engine module with its library loaded; fails loudly when the
    library or the device is missing (no fallback)."""
    from anukulan_b200 import pdhg
    pdhg.lib()
    assert pdhg.device_count() > 0, "no CUDA device visible to the engine"
    return pdhg
