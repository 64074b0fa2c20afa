import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running parity case")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    """Native libraries built in-tree (the product library and the oracle)."""
    from lare3d_b200 import build as b
    b.build()
    from oracle import oracle
    oracle.build()
    return True


STATE = ["rho", "energy", "vx", "vy", "vz", "bx", "by", "bz"]


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def interior(arr, lo, n, stag=0):
    """Slice Fortran indices 1..n (cells) or 0..n (nodes/faces) of an array
    whose lower bounds are lo."""
    sl = []
    for d in range(3):
        a = (1 if stag == 0 else 0) - lo[d]
        b = n[d] - lo[d] + 1
        sl.append(slice(a, b))
    return arr[tuple(sl)]
