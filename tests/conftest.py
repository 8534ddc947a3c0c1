import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_engine():
    from vldb_voila_b200 import Engine
    return Engine(0)


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
