import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: longer CPU or GPU runs")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gpu_lib():
    """Built CUDA library; GPU tests fail (not skip) when it is missing."""
    from cosenu_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from cosenu_b200.build import build
        build()
    return _lib.load()
