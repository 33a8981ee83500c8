"""Allocation-free entry point dazi_dk_iso_noalloc_dev.

It exists for callers that cannot let the library call cudaMalloc (a driver
living under another framework's allocator or a fixed device-memory budget,
or a pipeline that must avoid cudaMalloc's device-wide synchronisation).  The
caller passes device inputs and outputs; the library's only other device
memory is a static array.  These tests call it through the C-ABI, with the
library's own ctypes binding, and check its results against the existing
device entry dazi_dk_iso_dev (plain form) with the tolerances of the other
plain-form tests:
  - twice in a row on two different inputs, checking that the second call
    leaves the device's free memory unchanged;
  - on a grid whose columns need more than one tile of the static array
    (200 nodes x 160 periods: 21 columns per tile), so the tile loop runs;
  - with sen_* NULL, where only each column's base model runs.
Collected last on purpose, so a failure here cannot hide another test's
result."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from dazi_current_release_b200 import _lib
from dazi_current_release_b200 import synthetic as S

pytestmark = pytest.mark.gpu

NOALLOC_FLOATS = 4 << 20      # the static array's size in floats


def _dev_inputs(case, torch, dev):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev)  # noqa: E731
    return (t(case.vel), torch.from_numpy(case.periods.copy()).to(dev),
            torch.from_numpy(case.depz.copy()).to(dev))


def _outputs(nxy, K, nz, torch, dev, kernels=True):
    pv = torch.full((nxy * K,), -1.0, dtype=torch.float64, device=dev)
    sen = [torch.full((nxy * K * nz,), -1.0, dtype=torch.float64, device=dev)
           for _ in range(3)] if kernels else None
    st = torch.full((nxy,), -1, dtype=torch.int32, device=dev)
    return pv, sen, st


def _call(noalloc, case, ins, outs, torch):
    """One call through the C-ABI: the allocation-free entry, or
    dazi_dk_iso_dev in the plain form.  Returns host copies of pv, the
    three kernels (or None) and the statuses."""
    L = _lib.load()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    vel, per, depz = ins
    pv, sen, st = outs
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    ks = [P(s) for s in sen] if sen is not None else [None, None, None]
    head = (nx, ny, nz, P(vel), None, None, P(pv), *ks, K, P(per), P(depz),
            ctypes.c_float(case.minthk), 1, nx * ny)
    if noalloc:
        rc = L.dazi_dk_iso_noalloc_dev(*head, P(st), None)
    else:
        rc = L.dazi_dk_iso_dev(*head, _lib.FORM_PLAIN, P(st), None)
    assert rc == 0, L.dazi_dk_last_error()
    torch.cuda.synchronize()
    return (pv.cpu().numpy(), None if sen is None else [s.cpu().numpy() for s in sen],
            st.cpu().numpy())


def _compare(got, ref, case):
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    np.testing.assert_array_less(np.abs(got[0] / ref[0] - 1.0), 1e-6)
    np.testing.assert_array_equal(got[2], ref[2])
    if got[1] is None:
        return
    for g, r in zip(got[1], ref[1]):
        g = g.reshape(nx * ny, K * nz, order="F")
        r = r.reshape(nx * ny, K * nz, order="F")
        assert max(rel_l2(g[c], r[c]) for c in range(nx * ny)) <= 1e-4


def _deep_grid(nx, ny, seed, nz=200, K=160):
    """nz nodes 0.3-1.2 km apart (one sublayer each at minthk 0.5, so 200
    refined layers at nz = 200), a Vs gradient with 3 % noise, K periods."""
    rng = np.random.default_rng(seed)
    dep = np.concatenate([[0.0], np.cumsum(rng.uniform(0.3, 1.2, nz - 1))]).astype(np.float32)
    grad = 2.6 + 2.0 * dep / dep[-1]
    vel = (grad[None, None, :] * (1.0 + 0.03 * rng.standard_normal((nx, ny, nz))))
    return S.GridCase("deep", np.asfortranarray(vel.astype(np.float32)), dep,
                      np.geomspace(2.0, 100.0, K), 0.5)


def test_noalloc_matches_allocating_entry_on_two_calls():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    full = S.config1()
    cases = [S.subgrid(full, 5, 4), S.subgrid(S.config0(), 4, 4)]
    cases[1].vp = cases[1].rho = None     # Brocher path for both
    for n, case in enumerate(cases):
        nx, ny, nz = case.vel.shape
        K = case.periods.size
        ins = _dev_inputs(case, torch, dev)
        ref = _call(False, case, ins, _outputs(nx * ny, K, nz, torch, dev), torch)
        outs = _outputs(nx * ny, K, nz, torch, dev)
        if n == 1:
            free_before = torch.cuda.mem_get_info(dev)[0]
        got = _call(True, case, ins, outs, torch)
        if n == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        _compare(got, ref, case)


def test_noalloc_runs_several_tiles():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    case = _deep_grid(5, 5, seed=21)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    per_tile = NOALLOC_FLOATS // ((1 + 6 * nz) * K)
    assert per_tile == 21 and nx * ny > per_tile      # two launches: 21 + 4 columns
    ins = _dev_inputs(case, torch, dev)
    ref = _call(False, case, ins, _outputs(nx * ny, K, nz, torch, dev), torch)
    got = _call(True, case, ins, _outputs(nx * ny, K, nz, torch, dev), torch)
    _compare(got, ref, case)


def test_noalloc_phase_velocities_only():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    case = S.subgrid(S.config1(), 6, 5)
    case.vp = case.rho = None
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    ins = _dev_inputs(case, torch, dev)
    ref = _call(False, case, ins, _outputs(nx * ny, K, nz, torch, dev), torch)
    for _ in range(2):
        got = _call(True, case, ins, _outputs(nx * ny, K, nz, torch, dev, kernels=False), torch)
        _compare(got, ref, case)


def test_noalloc_rejects_oversize_and_bad_input():
    torch = pytest.importorskip("torch")
    f = _lib.load().dazi_dk_iso_noalloc_dev
    dev = torch.device("cuda", 0)
    z = torch.zeros(8, dtype=torch.float64, device=dev)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    # nz beyond the compiled limit
    assert f(2, 2, 201, P(z), None, None, P(z), None, None, None, 2, P(z), P(z),
             ctypes.c_float(4.0), 1, 4, None, None) == _lib.DAZI_ERR_LIMITS
    # column range outside the grid
    assert f(2, 2, 3, P(z), None, None, P(z), None, None, None, 2, P(z), P(z),
             ctypes.c_float(4.0), 3, 4, None, None) == _lib.DAZI_ERR_BADARG
