"""Shared test setup: the gpu marker, import paths and the oracle build."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    from build_oracle import build_oracle
    build_oracle()
    yield


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
