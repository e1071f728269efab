import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native sm_100a path")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def native_lib():
    from cccollisions_b200 import build
    build.build()
    from cccollisions_b200 import _native
    return _native.lib()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cccollisions_b200 import build
    build.build()
    return torch.device("cuda:0")


def random_mesh_soup(seed, nx=8, ny=8, noise=0.02, drop=0.05, dtype=np.float64, fold=True):
    """Small jittered folded grid (see cccollisions_b200.workloads.jittered_fold)."""
    from cccollisions_b200 import workloads as W
    return W.jittered_fold(seed, nx, ny, noise, drop, dtype, fold)
