"""Love waves and group velocity (surfdisp96 iwave = 1, igr > 0).

1. The oracle against the reference's own Python surf96 (pDSurfTomo's
   Numba translation, golden vectors in tests/golden/surf96_wave.npz made by
   tests/golden/make_surf96_wave.py): an independent implementation of the
   same algorithm, so agreement is within the root tolerance.
2. The library's root_kernel instantiations for Love / group velocity,
   compiled for the host by tests/host_emu, against the oracle on uneven
   (config-3 recipe) and high-contrast random columns.

Tolerances.  Each root search stops when its bracket is narrower than
1e-6 c (surfdisp96.f:608), so two searches of the same zero end at most
2e-6 c apart.  Group velocity U = (1/t1a - 1/t1b) / (1/(t1a c0) - 1/(t1b c1))
with t1a,b = t/(1 -+ h), h = 0.005: moves of 2e-6 c in c0 and c1 move U by
at most 2 * 2e-6 / (2h) * (U/c) ~ 4e-4 U for normal dispersion (U < c)."""
import numpy as np
import pytest

from dazi_current_release_b200 import synthetic as S
from edge_models import _batch, _random_columns
from host_emu import emu

PHASE_MOVE = 2.0e-6
GROUP_MOVE = 4.0e-4
COMBOS = [(2, 0), (2, 1), (1, 0), (1, 1)]


def _golden():
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return np.load(os.path.join(here, "golden", "surf96_wave.npz"))


@pytest.mark.parametrize("iwave,igr", COMBOS)
def test_oracle_matches_reference_surf96(oracle, iwave, igr):
    g = _golden()
    off, L, t = g["layer_off"], g["layers"], g["periods"]
    ref = g[f"cg_ifunc{iwave}_itype{igr}"]
    got = np.zeros_like(ref)
    for j in range(ref.shape[0]):
        d, a, b, r = (L[q, off[j]:off[j + 1]] for q in range(4))
        got[j], st, _ = oracle.surfdisp96(d, a, b, r, t, iwave=iwave, igr=igr)
        assert st == 0
    rel = np.abs(got / ref - 1)
    if igr == 0:
        # roots within the tolerance; real*4 model arrays here, real*8 there
        assert rel.max() <= PHASE_MOVE
    else:
        assert rel.max() <= GROUP_MOVE
        assert np.median(rel) <= 1.0e-4


def test_love_differs_from_rayleigh_beyond_the_tolerance(oracle):
    """The fixtures separate the wave types (a density or secular-function
    mix-up would not pass the test above)."""
    g = _golden()
    assert np.abs(g["cg_ifunc1_itype0"] / g["cg_ifunc2_itype0"] - 1).min() > 1e-2
    # group = phase only where dc/dT = 0
    assert np.median(np.abs(g["cg_ifunc2_itype1"] / g["cg_ifunc2_itype0"] - 1)) > 1e-2
    assert np.median(np.abs(g["cg_ifunc1_itype1"] / g["cg_ifunc1_itype0"] - 1)) > 1e-2


def _oracle_batch(oracle, node_off, depz, vs, per_off, periods, minthk, iwave, igr):
    pv = np.zeros(int(per_off[-1]))
    status = []
    for c in range(len(node_off) - 1):
        n0, n1, p0, p1 = node_off[c], node_off[c + 1], per_off[c], per_off[c + 1]
        vp, rho = oracle.brocher(vs[n0:n1])
        thk, rvp, rvs, rrho, _ = oracle.refine(minthk, depz[n0:n1], vp, vs[n0:n1], rho)
        cg, st, _ = oracle.surfdisp96(thk, rvp, rvs, rrho, periods[p0:p1], iwave=iwave, igr=igr)
        pv[p0:p1] = cg
        status.append(st)
    return pv, np.array(status, np.int32)


def _cases():
    b = S.config3(realisations=1, columns=240, base_seed=1000)
    yield "uneven", (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    yield "random", (*_batch(_random_columns(120, seed=3)), 2.0)


@pytest.mark.parametrize("iwave,igr", COMBOS)
def test_root_kernel_matches_oracle(oracle, iwave, igr):
    for name, args in _cases():
        rc, pv, st, _ = emu.root_batch(*args, scan32=False, ifunc=1 if iwave == 1 else 2,
                                       group=igr > 0)
        ref, rst = _oracle_batch(oracle, *args, iwave, igr)
        assert rc == 0
        pv = pv[:ref.size]
        np.testing.assert_array_equal(st[:rst.size], rst, err_msg=name)
        moved = np.nonzero(pv != ref)[0]
        # Love evaluates dltar1 with the reference's operation order: exact
        if iwave == 1:
            assert moved.size == 0, (name, moved[:5])
        assert moved.size <= 0.05 * ref.size, (name, moved.size)
        bound = GROUP_MOVE if igr else PHASE_MOVE
        assert np.all(ref[moved] > 0)
        assert np.all(np.abs(pv[moved] / ref[moved] - 1) <= bound), name
