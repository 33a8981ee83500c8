"""Allocation-free entry point dazi_dk_iso_noalloc_dev.

It exists for callers that cannot let the library call cudaMalloc (a driver
living under another framework's allocator or a fixed device-memory budget,
or a pipeline that must avoid cudaMalloc's device-wide synchronisation).  The
caller passes device inputs and outputs; the library's only other device
memory is a static array.  This test calls it through the C-ABI twice in a
row, on two different inputs, and checks each result against the existing
device entry dazi_dk_iso_dev (plain form) with the tolerances of the other
plain-form tests; it also checks that the second call leaves the device's free
memory unchanged.  Collected last on purpose, so a failure here cannot hide
another test's result."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from dazi_current_release_b200 import _lib
from dazi_current_release_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _dev_inputs(case, torch, dev):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev)  # noqa: E731
    return (t(case.vel), torch.from_numpy(case.periods.copy()).to(dev),
            torch.from_numpy(case.depz.copy()).to(dev))


def _outputs(nxy, K, nz, torch, dev):
    pv = torch.full((nxy * K,), -1.0, dtype=torch.float64, device=dev)
    sen = [torch.full((nxy * K * nz,), -1.0, dtype=torch.float64, device=dev) for _ in range(3)]
    st = torch.full((nxy,), -1, dtype=torch.int32, device=dev)
    return pv, sen, st


def _call(fn, case, ins, outs, torch):
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    vel, per, depz = ins
    pv, sen, st = outs
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    rc = fn(nx, ny, nz, P(vel), None, None, P(pv), P(sen[0]), P(sen[1]), P(sen[2]), K, P(per),
            P(depz), ctypes.c_float(case.minthk), 1, nx * ny, _lib.FORM_PLAIN, P(st), None) \
        if fn.__name__ == "dazi_dk_iso_dev" else \
        fn(nx, ny, nz, P(vel), None, None, P(pv), P(sen[0]), P(sen[1]), P(sen[2]), K, P(per),
           P(depz), ctypes.c_float(case.minthk), 1, nx * ny, P(st), None)
    assert rc == 0, _lib.load().dazi_dk_last_error()
    torch.cuda.synchronize()
    return pv.cpu().numpy(), [s.cpu().numpy() for s in sen], st.cpu().numpy()


def _noalloc(L):
    f = L.dazi_dk_iso_noalloc_dev
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 7 + \
        [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_int,
         ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_matches_allocating_entry_on_two_calls():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    L = _lib.load()
    f_new = _noalloc(L)
    f_old = L.dazi_dk_iso_dev
    full = S.config1()
    cases = [S.subgrid(full, 5, 4), S.subgrid(S.config0(), 4, 4)]
    cases[1].vp = cases[1].rho = None     # Brocher path for both
    free_after_first = None
    for n, case in enumerate(cases):
        nx, ny, nz = case.vel.shape
        K = case.periods.size
        ins = _dev_inputs(case, torch, dev)
        ref = _call(f_old, case, ins, _outputs(nx * ny, K, nz, torch, dev), torch)
        outs = _outputs(nx * ny, K, nz, torch, dev)
        if n == 1:
            free_before = torch.cuda.mem_get_info(dev)[0]
        got = _call(f_new, case, ins, outs, torch)
        if n == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        np.testing.assert_array_less(np.abs(got[0] / ref[0] - 1.0), 1e-6)
        for g, r in zip(got[1], ref[1]):
            g = g.reshape(nx * ny, K * nz, order="F")
            r = r.reshape(nx * ny, K * nz, order="F")
            assert max(rel_l2(g[c], r[c]) for c in range(nx * ny)) <= 1e-4
        np.testing.assert_array_equal(got[2], ref[2])


def test_noalloc_rejects_oversize_and_bad_input():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    f = _noalloc(L)
    dev = torch.device("cuda", 0)
    z = torch.zeros(8, dtype=torch.float64, device=dev)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    # nz beyond the compiled limit
    assert f(2, 2, 201, P(z), None, None, P(z), None, None, None, 2, P(z), P(z),
             ctypes.c_float(4.0), 1, 4, None, None) == _lib.DAZI_ERR_LIMITS
    # column range outside the grid
    assert f(2, 2, 3, P(z), None, None, P(z), None, None, None, 2, P(z), P(z),
             ctypes.c_float(4.0), 3, 4, None, None) == _lib.DAZI_ERR_BADARG
