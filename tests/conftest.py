import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the libpartia_b200 kernels)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the CUDA library (nvcc cross-compiles without a GPU) and the CPU oracle if a
    fresh checkout has neither; on a GPU box both arrive prebuilt."""
    from distorteddustydiscanalysistoolkits_b200 import _build, _lib
    if not os.path.exists(_lib.LIB_PATH):
        _build.build()
    import oracle
    oracle.lib()
    yield


@pytest.fixture(scope="session")
def backend():
    import distorteddustydiscanalysistoolkits_b200 as pb
    b = pb.CUDAComputeBackend(0)
    yield b
    b.close()
