import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200); runs the CUDA engine")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture(scope="session")
def corr_small(golden):
    import scipy.sparse as sp
    k = golden("krylov.npz")
    n = k["corr_indptr"].size - 1
    return sp.csr_matrix((k["corr_data"], k["corr_indices"], k["corr_indptr"]),
                         shape=(n, n))


@pytest.fixture(scope="session")
def cuda():
    """The engine library on a CUDA device (GPU tests only)."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is available")
    from imate_b200 import _build, _lib
    _build.build()
    return _lib.load()
