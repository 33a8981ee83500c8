import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU-oracle runs")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    O.lib()
    return O


@pytest.fixture(scope="session")
def yunnan():
    d = np.load(os.path.join(GOLDEN, "yunnan_pv.npz"))
    return {k: d[k] for k in d.files}


def inner_columns(pv, nx, ny):
    """tRcV((jj-1)*(nx-2)+ii,k) = pvRc(jj*nx+ii+1,k), CalSurfG_parallel.f90:2519-2527,
    flattened in the WTPeriodPhaseV print order (period, jj, ii)."""
    K = pv.shape[1]
    jj, ii = np.meshgrid(np.arange(1, ny - 1), np.arange(1, nx - 1), indexing="ij")
    idx = (jj * nx + ii).ravel()
    return np.concatenate([pv[idx, k] for k in range(K)])


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)
