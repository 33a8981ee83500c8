"""GPU LSMR (dazi_lsmr_dev / dazi_lsmr) against the reference's SciPy
backend of its LSMR call (oracle/lsmr_ref.py: scipy.sparse.linalg.lsmr on
the same triplets, as code/depthkernel_lab/scipy_lsmr_triplet_solver.py
runs it), on a G-like system (tests/lsmr_systems.py).

LSMR's iterates on this system are sensitive to rounding once the
bidiagonalisation loses orthogonality: SciPy against itself with b changed
by 1e-15 relative differs by 8e-6 in x after 20 iterations, and an exact
re-arrangement of the same arithmetic differs from SciPy by 1.8e-4 after
50.  So:
- the first iterations (5 and 10, all tolerances 0) must agree with SciPy
  to 1e-12 and 1e-9 in x and in every estimate;
- converged solves (damp 0 and 0.2, atol = btol = 1e-6, conlim 1e8) must
  stop by the same rule within two iterations, with ||r|| within 1e-6, and
  lie as close to the fully converged solution (SciPy at atol = btol =
  1e-15) as SciPy's own solve does (within 1.5x + 1e-6; both are about
  3e-5 from it);
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


@pytest.mark.parametrize("iters,tol", [(5, 1e-12), (10, 1e-9)])
def test_first_iterations_match_scipy(system, iters, tol):
    torch = pytest.importorskip("torch")
    row, col, val, b, m, n = system
    r = lsmr(*_dev(torch, row, col, val, b), m, n, atol=0.0, btol=0.0, conlim=0.0,
             maxiter=iters)
    ref = lsmr_ref.lsmr(row, col, val, b, m, n, atol=0.0, btol=0.0, conlim=0.0, maxiter=iters)
    assert (r.istop, r.itn) == (7, iters) == (ref[1], ref[2])
    assert _rel(r.x.cpu().numpy(), ref[0]) <= tol
    for got, exp in ((r.normr, ref[3]), (r.normAr, ref[4]), (r.normA, ref[5]), (r.condA, ref[6]),
                     (r.normx, ref[7])):
        assert abs(got - exp) <= tol * abs(exp)


@pytest.mark.parametrize("damp", [0.0, 0.2])
def test_converged_solve_as_accurate_as_scipy(system, damp):
    torch = pytest.importorskip("torch")
    row, col, val, b, m, n = system
    r = lsmr(*_dev(torch, row, col, val, b), m, n, damp=damp, atol=1e-6, btol=1e-6, conlim=1e8)
    ref = lsmr_ref.lsmr(row, col, val, b, m, n, damp=damp, atol=1e-6, btol=1e-6, conlim=1e8)
    best = lsmr_ref.lsmr(row, col, val, b, m, n, damp=damp, atol=1e-15, btol=1e-15, conlim=0.0,
                         maxiter=5000)[0]
    x = r.x.cpu().numpy()
    e_gpu, e_ref = _rel(x, best), _rel(ref[0], best)
    print(f"damp {damp}: GPU istop {r.istop} itn {r.itn} error {e_gpu:.2e}; SciPy istop "
          f"{ref[1]} itn {ref[2]} error {e_ref:.2e}; x apart {_rel(x, ref[0]):.2e}")
    assert r.istop == ref[1] and abs(r.itn - ref[2]) <= 2
    assert abs(r.normr - ref[3]) <= 1e-6 * ref[3]
    assert e_gpu <= 1.5 * e_ref + 1e-6


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
