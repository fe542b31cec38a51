"""Shared test setup: import paths for the library binding and the oracle, the `gpu` marker."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "alias-table-gpu_b200")
ORACLE = os.path.join(REPO, "oracle")
for p in (PKG, ORACLE, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; a GPU test fails (not skips) when there is none."""
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    import wrs
    assert wrs.lib().wrs_check_device() == 0, "device is not an sm_100 part"
    return torch.device("cuda:0")
