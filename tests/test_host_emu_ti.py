"""The library's Gc/Gs device code (table build + per-(column, period)
sweep), compiled for the host by tests/host_emu, against the oracle of
tregn96 / depthkernelTI on the CPU.  The same arithmetic runs on the GPU
(tests/test_gpu_ti.py, tests/test_gpu_batch.py check the device results);
this suite exercises it here on every kind of layer: evanescent,
oscillatory, complex-eigenvalue (config 4's deep layers at short periods)
and the half-space."""
import numpy as np
import pytest

from conftest import rel_l2
from dazi_current_release_b200 import synthetic as S
from edge_models import _batch, _random_columns, leaky_periods
from host_emu import emu


def _grid_as_batch(case):
    nx, ny, nz = case.vel.shape
    n = nx * ny
    K = case.periods.size
    node_off = np.arange(n + 1, dtype=np.int64) * nz
    per_off = np.arange(n + 1, dtype=np.int64) * K
    vs = case.vel.reshape(n, nz, order="F").ravel()
    return node_off, np.tile(case.depz, n), vs, per_off, np.tile(case.periods, n), case.minthk


def _compare(oracle, node_off, depz, vs, per_off, per, minthk, skip_leaky=False):
    ref = oracle.batch(node_off, depz, vs, per_off, per, minthk, kernels=False)
    rc, ls, ls_off = emu.ti_batch(node_off, depz, vs, per_off, per, minthk, ref["pv"])
    assert rc == 0
    worst = 0.0
    for c in range(node_off.size - 1):
        K = int(per_off[c + 1] - per_off[c])
        nz = int(node_off[c + 1] - node_off[c])
        got = ls[ls_off[c]:ls_off[c + 1]].reshape((K, nz - 1), order="F")
        exp = ref["lsen"][ls_off[c]:ls_off[c + 1]].reshape((K, nz - 1), order="F")
        keep = np.ones(K, bool)
        if skip_leaky:
            keep = ~leaky_periods(ref["pv"][per_off[c]:per_off[c + 1]], vs[node_off[c + 1] - 1],
                                  oracle.brocher)
        if keep.any():
            e = rel_l2(got[keep], exp[keep])
            worst = max(worst, e)
            assert e <= 1e-5, (c, e)
            assert np.abs(got[keep] - exp[keep]).max() <= 1e-4, c
    return worst


@pytest.mark.parametrize("make", [lambda: S.subgrid(S.config1(), 4, 3),
                                  lambda: S.subgrid(S.config4(), 3, 2)])
def test_grid_columns(oracle, make):
    worst = _compare(oracle, *_grid_as_batch(make()))
    print("worst per-column rel-L2", worst)


def test_uneven_columns(oracle):
    b = S.config3(realisations=1, columns=200, base_seed=1000)
    worst = _compare(oracle, b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    print("worst per-column rel-L2", worst)


def test_random_edge_columns(oracle):
    node_off, depz, vs, per_off, per = _batch(_random_columns(60))
    worst = _compare(oracle, node_off, depz, vs, per_off, per, 2.0, skip_leaky=True)
    print("worst per-column rel-L2", worst)
