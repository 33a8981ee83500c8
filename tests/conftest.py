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


def assert_pv_parity(got, ref, ref_unrounded, midpoint_rel=1e-8, allow_tol_moves=False,
                     tol=1.0e-6):
    """Phase velocities against the oracle: bit-identical, except
      - a root whose unrounded double value lies within midpoint_rel
        (relative) of a float32 rounding midpoint may round to the
        neighbouring float32 (the reference stores sngl(c),
        surfdisp96.f:292-297; any last-bit difference of the double
        arithmetic flips such a root);
      - with allow_tol_moves, a root that moved within the root search's
        own convergence tolerance (|c1 - c2| <= tol * c1, surfdisp96.f:608):
        a Neville step at a point where F is zero to FP64 rounding can take
        the other branch and end elsewhere in the final bracket.
    Returns the number of differing values."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    ru = np.asarray(ref_unrounded, np.float64)
    diff = np.nonzero(got != ref)[0]
    for k in diff:
        f = np.float32(ref[k])
        one_ulp = np.float32(got[k]) in (np.nextafter(f, np.float32(np.inf)),
                                         np.nextafter(f, np.float32(-np.inf)))
        mid = (float(f) + float(np.float32(got[k]))) / 2
        if one_ulp and abs(ru[k] - mid) / abs(ru[k]) <= midpoint_rel:
            continue
        assert allow_tol_moves, f"pv[{k}] = {got[k]!r}, oracle {ref[k]!r}: not a rounding flip"
        assert ref[k] > 0 and abs(got[k] - ref[k]) <= tol * ref[k], \
            f"pv[{k}] = {got[k]!r}, oracle {ref[k]!r}: beyond the root tolerance"
    return diff.size


def assert_fd_parity(got, exp, x, dln=0.01, max_frac=0.02, tol=1.0e-6, cmax=8.0):
    """Finite-difference kernels (K, nz) against the oracle's: equal, except
    a few entries whose perturbed-model roots differ from the oracle's
    within the root search's own convergence tolerance (|c1 - c2| <=
    tol * c1, surfdisp96.f:608): a root on a float32 rounding midpoint (see
    assert_pv_parity), or a Neville sequence that took another branch at a
    point where F is zero to FP64 rounding.  Bound on the difference
    quotient: |d| * dln * x_i <= 2 tol cmax.  x: the perturbed node values
    (Vs, Vp or rho).  Returns the number of differing entries."""
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    d = np.abs(got - exp) * dln * np.asarray(x, np.float64)[None, :]
    n = int(np.count_nonzero(got != exp))
    assert (d <= 2.0 * tol * cmax).all(), f"FD kernel differs by {d.max():.3g} km/s in the difference"
    assert n <= max(2, max_frac * got.size), f"{n} of {got.size} FD entries differ"
    return n
