import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "oracle"), os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests fail, not skip, without a GPU: a skipped parity test would
    hide a missing native path."""
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from pymonteopt_b200 import _lib
    _lib.load()
    return torch.device("cuda", 0)
