import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) CUDA device")


@pytest.fixture(scope="session")
def engine():
    """One al_engine on cuda:0 for the whole GPU session."""
    import torch
    from alluvion_b200 import _capi
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    eng = _capi.Engine(0)
    yield eng
    eng.close()


def dev(a):
    """Host numpy array -> CUDA torch tensor (same dtype, contiguous)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()
