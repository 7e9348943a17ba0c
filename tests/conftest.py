import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device and the built spider_b200 library")


def _cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    if not _cuda_ok():
        pytest.skip("no CUDA device")
    from spider_b200 import ops
    c = ops.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
