"""Shared fixtures. `gpu`-marked tests need a CUDA device (B200) and the built
native library; the rest run on CPU only."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built sm_100a library")


@pytest.fixture(scope="session")
def gf():
    import __graft_entry__
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
