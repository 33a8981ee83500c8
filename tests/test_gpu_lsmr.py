"""GPU LSMR (dazi_lsmr_dev / dazi_lsmr) against the reference's SciPy
backend of its LSMR call (oracle/lsmr_ref.py: scipy.sparse.linalg.lsmr on
the same triplets, as code/depthkernel_lab/scipy_lsmr_triplet_solver.py
runs it), on G-like systems (tests/lsmr_systems.py):

- converged solves (damp 0 and 0.2, atol = btol = 1e-6, conlim 1e8): the
  same stopping rule, the same iteration count within one, x and the
  norm estimates within 1e-6;
- a fixed number of iterations (all tolerances 0, 50 iterations): x and the
  estimates within 1e-9 (the two differ only in summation order);
- the Fortran-shaped host entry (iw = rows then columns, rw = values)
  gives the device entry's x bit for bit;
- a zero right-hand side stops at once with x = 0; an index outside the
  matrix is rejected."""
import ctypes

import numpy as np
import pytest

from lsmr_systems import g_like_system
from oracle import lsmr_ref
from dazi_current_release_b200 import _lib
from dazi_current_release_b200.lsmr import lsmr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    return g_like_system()


def _dev(torch, row, col, val, b):
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    return t(row), t(col), t(val), t(b)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("damp", [0.0, 0.2])
def test_converged_solve_matches_scipy(system, damp):
    torch = pytest.importorskip("torch")
    row, col, val, b, m, n = system
    r = lsmr(*_dev(torch, row, col, val, b), m, n, damp=damp, atol=1e-6, btol=1e-6, conlim=1e8)
    ref = lsmr_ref.lsmr(row, col, val, b, m, n, damp=damp, atol=1e-6, btol=1e-6, conlim=1e8)
    x = r.x.cpu().numpy()
    print(f"damp {damp}: GPU istop {r.istop} itn {r.itn}; SciPy istop {ref[1]} itn {ref[2]}; "
          f"x rel {_rel(x, ref[0]):.2e}")
    assert r.istop == ref[1] and abs(r.itn - ref[2]) <= 1
    assert _rel(x, ref[0]) <= 1e-6
    for got, exp in ((r.normr, ref[3]), (r.normAr, ref[4]), (r.normA, ref[5]), (r.normx, ref[7])):
        assert abs(got - exp) <= 1e-6 * abs(exp) + 1e-12


def test_fixed_iterations_match_scipy(system):
    torch = pytest.importorskip("torch")
    row, col, val, b, m, n = system
    r = lsmr(*_dev(torch, row, col, val, b), m, n, atol=0.0, btol=0.0, conlim=0.0, maxiter=50)
    ref = lsmr_ref.lsmr(row, col, val, b, m, n, atol=0.0, btol=0.0, conlim=0.0, maxiter=50)
    assert (r.istop, r.itn) == (7, 50) == (ref[1], ref[2])
    assert _rel(r.x.cpu().numpy(), ref[0]) <= 1e-9
    for got, exp in ((r.normr, ref[3]), (r.normAr, ref[4]), (r.normA, ref[5]), (r.condA, ref[6]),
                     (r.normx, ref[7])):
        assert abs(got - exp) <= 1e-9 * abs(exp)


def test_fortran_entry_equals_device_entry(system):
    torch = pytest.importorskip("torch")
    row, col, val, b, m, n = system
    r = lsmr(*_dev(torch, row, col, val, b), m, n, damp=0.1, maxiter=40)
    L = _lib.load()
    iw = np.concatenate([row, col]).astype(np.int32)
    x = np.zeros(n)
    ci, cl, cd = ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    istop, itn = ci(0), ci(0)
    outs = [cd(0.0) for _ in range(5)]
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    rc = L.dazi_lsmr(ctypes.byref(ci(m)), ctypes.byref(ci(n)), ctypes.byref(cl(iw.size)),
                     ctypes.byref(cl(val.size)), P(iw, ci), P(val, ctypes.c_float),
                     P(np.ascontiguousarray(b), cd), ctypes.byref(cd(0.1)), ctypes.byref(cd(1e-6)),
                     ctypes.byref(cd(1e-6)), ctypes.byref(cd(1e8)), ctypes.byref(ci(40)),
                     ctypes.byref(ci(0)), ctypes.byref(ci(6)), P(x, cd), ctypes.byref(istop),
                     ctypes.byref(itn), *[ctypes.byref(o) for o in outs])
    assert rc == 0, L.dazi_dk_last_error()
    np.testing.assert_array_equal(x, r.x.cpu().numpy())
    assert (istop.value, itn.value) == (r.istop, r.itn)
    assert outs[0].value == r.normA and outs[4].value == r.normx


def test_zero_rhs_and_bad_index(system):
    torch = pytest.importorskip("torch")
    row, col, val, b, m, n = system
    r = lsmr(*_dev(torch, row, col, val, np.zeros_like(b)), m, n)
    assert r.istop == 0 and r.itn == 0
    assert not r.x.abs().max().item()
    bad = col.copy()
    bad[7] = n + 1
    with pytest.raises(_lib.DaziError) as ei:
        lsmr(*_dev(torch, row, bad, val, b), m, n)
    assert ei.value.code == _lib.DAZI_ERR_BADARG
