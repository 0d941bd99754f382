"""Shared test setup.  `-m gpu` tests need a B200 and the built libzkgpu.so;
everything else runs on CPU against the oracle (oracle/) only."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libzkgpu.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def zk():
    import zk_gpu_b200
    zk_gpu_b200.lib()
    return zk_gpu_b200
