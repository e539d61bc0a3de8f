"""Shared test settings: the gpu marker, devices, and the synthetic networks."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (a B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("this test needs a GPU")
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def networks():
    from maxichem_b200 import synthetic

    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = synthetic.network(name)
        return cache[name]

    return get
