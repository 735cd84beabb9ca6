import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    O.lib()
    return O


@pytest.fixture(scope="session")
def neat():
    """The CUDA library (built in-tree); GPU tests fail loudly without it."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from neat_b200.csrc import build
    build.build()
    from neat_b200 import _lib
    return _lib.load()
