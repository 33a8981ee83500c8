"""G-row epilogue (sparse rows of the LSMR system from the kernels) on the
GPU against the oracle of CalSurfG_parallel.f90:2363-2400, bit for bit:
same entries, values, row ids, parameter columns and order."""
import numpy as np
import pytest

from dazi_current_release_b200 import _lib
from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.grows import g_rows

pytestmark = pytest.mark.gpu


def _rays(nvx, nvz, K, nrays, seed=3):
    rng = np.random.default_rng(seed)
    ncell = nvx * nvz
    cells, off = [], [0]
    for _ in range(nrays):
        n = int(rng.integers(1, ncell + 1))
        cells.append(np.sort(rng.choice(ncell, n, replace=False)))
        off.append(off[-1] + n)
    cell = np.concatenate(cells).astype(np.int32)
    fdm = (rng.lognormal(-1.0, 2.0, cell.size) * rng.choice([-1, 1], cell.size)).astype(np.float32)
    fdm[rng.random(cell.size) < 0.1] = 3e-5                  # below ftol: cell skipped
    th = rng.uniform(0, np.pi, cell.size)
    fdmc = (fdm * np.cos(2 * th)).astype(np.float32)
    fdms = (fdm * np.sin(2 * th)).astype(np.float32)
    per = rng.integers(0, K, nrays).astype(np.int32)
    rid = (np.arange(nrays) * 3 + 7).astype(np.int32)
    return per, rid, np.asarray(off, np.int64), cell, fdm, fdmc, fdms


def _inputs(oracle):
    case = S.subgrid(S.config1(), 6, 5)                      # 4 x 3 inner cells
    nx, ny, nz = case.vel.shape
    ref = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk)
    ti = oracle.depthkernel_ti(case.vel, case.depz, case.periods, case.minthk)
    return case, ref, ti


@pytest.mark.parametrize("aniso", [True, False])
def test_grows_match_oracle(oracle, aniso):
    case, ref, ti = _inputs(oracle)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    per, rid, off, cell, fdm, fdmc, fdms = _rays(nx - 2, ny - 2, K, 60)
    ls = ti["Lsen_Gsc"] if aniso else None
    args = (case.vel, ref["sen_vs"], ref["sen_vp"], ref["sen_rho"], ls, per, rid, off, cell, fdm,
            fdmc if aniso else None, fdms if aniso else None)
    rw, iw, col, nnz = g_rows(*args)
    erw, eiw, ecol, ennz = oracle.grows(nx - 2, ny - 2, *args)
    print("entries", rw.size, "of", off[-1] * (nz - 1) * (3 if aniso else 1), "candidates")
    assert rw.size > 0
    np.testing.assert_array_equal(nnz, ennz)
    np.testing.assert_array_equal(col, ecol)
    np.testing.assert_array_equal(iw, eiw)
    np.testing.assert_array_equal(rw, erw)


def test_grows_capacity_and_bad_rays(oracle):
    case, ref, ti = _inputs(oracle)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    per, rid, off, cell, fdm, fdmc, fdms = _rays(nx - 2, ny - 2, K, 10)
    args = [case.vel, ref["sen_vs"], ref["sen_vp"], ref["sen_rho"], ti["Lsen_Gsc"], per, rid, off,
            cell, fdm, fdmc, fdms]
    with pytest.raises(_lib.DaziError) as e:
        g_rows(*args, cap=5)
    assert e.value.code == _lib.DAZI_ERR_LIMITS
    bad = cell.copy()
    bad[off[1] - 1], bad[off[1] - 2] = bad[off[1] - 2], bad[off[1] - 1]  # not ascending
    args[8] = bad
    if off[1] - off[0] >= 2:
        with pytest.raises(_lib.DaziError) as e:
            g_rows(*args)
        assert e.value.code == _lib.DAZI_ERR_BADARG
