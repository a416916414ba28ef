import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size case, minutes of work")


def gpu_available() -> bool:
    try:
        import euplectella_hpc_b200 as E
        return E.device_count() > 0
    except ImportError:
        return False


@pytest.fixture(scope="session")
def eup():
    import euplectella_hpc_b200 as E
    return E


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture
def require_gpu(eup):
    if eup.device_count() == 0:
        pytest.fail("no CUDA device visible: -m gpu tests need a B200")


def fluid_mask_haloed(obs: np.ndarray) -> np.ndarray:
    """Boolean mask over the haloed array (n+2, m+2, l+2): True except interior solid voxels."""
    n, m, l = obs.shape
    keep = np.ones((n + 2, m + 2, l + 2), dtype=bool)
    keep[1:-1, 1:-1, 1:-1] = obs != 1
    return keep
