import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.build()
    return o


@pytest.fixture(scope="session")
def u26ctx():
    import torch
    from untangling26_b200 import Context
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    ctx = Context(0)
    yield ctx
    ctx.close()
