import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def hmg():
    import hmglib_b200
    from hmglib_b200 import build
    build.build()
    return hmglib_b200


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


def golden(name):
    import numpy as np
    p = os.path.join(ROOT, "tests", "golden", name + ".npz")
    if not os.path.exists(p):
        pytest.skip(f"golden fixture {name} not generated")
    return dict(np.load(p))
