import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import ats_oracle
    ats_oracle.build()
    return ats_oracle


@pytest.fixture(scope="session")
def ats():
    import libatssim_b200
    from libatssim_b200 import build
    build.build()
    return libatssim_b200


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
