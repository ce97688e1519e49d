"""pytest configuration: the `gpu` marker and the repository on sys.path."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libmfixgpu.so")


@pytest.fixture(scope="session")
def cuda():
    """torch with a visible GPU (device memory for the device-pointer entry points)."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a visible CUDA device")
    return torch
