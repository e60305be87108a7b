import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def gpu_lib():
    """The built CUDA library; a GPU test fails loudly if it is missing."""
    import torch
    assert torch.cuda.is_available(), "gpu test without a visible GPU"
    from frank_b200 import build
    build.build()
    from frank_b200._abi import lib
    return lib()
