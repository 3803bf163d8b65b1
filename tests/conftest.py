"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Build (incrementally) the CUDA library and the CPU checker."""
    from research_b200 import build
    build.build_cuda()
    build.build_passes()
    build.build_oracle()
    return True


@pytest.fixture(scope="session")
def rr(built):
    from research_b200 import rr as _rr
    return _rr


@pytest.fixture(scope="session")
def O(built):
    import oracle as _o
    return _o


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def ctx(rr, torch_cuda):
    c = rr.Context(0)
    yield c
    c.close()


def to_np(t):
    return t.detach().cpu().numpy()
