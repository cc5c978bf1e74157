"""Shared pytest setup: registers the `gpu` marker, puts the repository root on
sys.path (for `oracle` and `__graft_entry__`) and registers the package
directory cross-denoiser_b200 as the module cross_denoiser_b200."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import __graft_entry__  # noqa: E402

__graft_entry__.load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); run with -m gpu")


@pytest.fixture(scope="session")
def cd():
    return sys.modules["cross_denoiser_b200"]


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda:0")
