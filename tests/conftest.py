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
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle and (if missing) the product library once per session."""
    from oracle import oracle as orc
    orc.build()
    from signalalign_b200 import build as sab
    if not os.path.exists(sab.LIB):
        sab.build()
    yield
