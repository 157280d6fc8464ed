import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs libptb200 kernels)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (test infrastructure): built on first use."""
    from oracle import build, oracle as o
    build.build()
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test requested but no CUDA device is visible")
    from particle_transport_b200 import build as b
    if not os.path.exists(b.LIB):
        pytest.fail("libptb200.so is not built")
    return torch
