import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")
    config.addinivalue_line("markers", "slow: longer CPU tests")


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; GPU tests fail (not skip) without one, so a
    silent CPU run cannot pass them."""
    import torch
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    torch.cuda.init()
    return torch


def seeded(seed):
    return np.random.default_rng(seed)


# Parity tolerance: relative L2 against the oracle (the CPU restatement of
# the reference) and against the FP64 DFT, FP32 path.
REL_L2_TOL = 1e-5
