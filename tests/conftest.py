import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import cpu
    cpu.lib()
    return cpu


@pytest.fixture(scope="session")
def native_lib():
    """The native library, built in-tree if it is missing."""
    from cm_halofinder_b200 import _abi, build
    if not os.path.exists(_abi.LIB_PATH):
        build.build()
    return _abi.lib()
