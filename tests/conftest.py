import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def small_mesh():
    from src_b200 import mesh
    cm = mesh.generate(12, L=9, seed=3)
    return cm, cm.to_reference()


@pytest.fixture(scope="session")
def c1_mesh():
    """The small CPU-runnable workload: 48x48 jittered columns x 41 levels, hill h0=400 m."""
    from src_b200 import mesh
    cm = mesh.generate(48, L=41, seed=0, h0=400.0)
    return cm, cm.to_reference()


@pytest.fixture(scope="session")
def open_mesh():
    """Open channel (iper = 0): 12x12 columns from corner to corner of the 120 km square, 9
    levels, inflow at x = 0 (type 7), outflow at x = Lx (8), walls at y = 0 and y = Ly (5, 6)."""
    from src_b200 import mesh
    cm = mesh.generate(12, L=9, seed=5, periodic=False)
    return cm, cm.to_reference()
