import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

REFERENCE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the libpartia_b200 kernels)")


@pytest.fixture(scope="session")
def backend():
    import distorteddustydiscanalysistoolkits_b200 as pb
    b = pb.CUDAComputeBackend(0)
    yield b
    b.close()
