import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="session")
def golden_ops():
    return np.load(os.path.join(GOLDEN, "reference_ops.npz"))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle(4)


@pytest.fixture(scope="session")
def gpu_lib():
    """The built CUDA library on a machine with a GPU (skips otherwise is not
    allowed for gpu-marked tests: they fail loudly if the library is absent)."""
    import easybem_b200
    from easybem_b200 import _lib
    _lib.lib()
    return easybem_b200
