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
    """Small jittered grid folded over itself, with a random displacement (x0, x1, masses).

    Shared vertices are exact (soup built from an indexed mesh), so the shared-vertex rules
    are exercised.
    """
    from cccollisions_b200 import workloads as W
    g = np.random.Generator(np.random.PCG64(seed))
    v, f = W.grid(nx, ny)
    v[:, 2] = g.normal(0, noise, v.shape[0])
    if fold:
        m = v[:, 0] > 0.5
        v[m, 0] = 1.0 - v[m, 0]
        v[m, 2] += 0.01
    v1 = v.copy()
    v1[:, 2] -= drop
    v1 += g.normal(0, noise, v.shape)
    x0 = W.soup(v, f).astype(dtype)
    x1 = W.soup(v1, f).astype(dtype)
    masses = g.uniform(0.5, 2.0, (x0.shape[0], 3)).astype(dtype)
    return x0, x1, masses
