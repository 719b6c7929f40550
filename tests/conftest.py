import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device; runs the CUDA kernels")


@pytest.fixture(scope="session")
def cuda_device():
    """GPU tests must run on a device: fail (not skip) when none is usable."""
    import cpipe_b200
    n = cpipe_b200.lib().cpipe_cuda_device_count()
    assert n > 0, "no CUDA device visible; -m gpu tests need a B200"
    return n


@pytest.fixture(scope="session")
def host(cuda_device):
    from cpipe_b200 import Host
    h = Host()
    yield h
    h.close()


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name + ".npz"))
