import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_lib():
    """Loads the in-tree CUDA library; GPU tests fail (not skip) if it is missing."""
    import torch

    assert torch.cuda.is_available(), "GPU test run without a visible CUDA device"
    import fluxo_b200

    return fluxo_b200.load()
