"""The adjoint sweeps of the library (k_adjoint.cu: Rayleigh and Love, phase
and group velocity), compiled for the host by tests/host_emu and driven as
run_tables drives them, against the oracle on the CPU.

1. Phase velocity: against the oracle's exact-model central differences
   (double-precision model pipeline, root converged to 1e-13, dln = 1e-4),
   within 1e-5 rel-L2 per column, with the Rayleigh sweep's depth cut
   reached (the deepest node of some pairs is zero).
2. Group velocity, U = (1/t1a - 1/t1b) / (1/(t1a c0) - 1/(t1b c1)),
   t1a,b = t/(1 -+ h), h = 0.005: against the same differences of the
   oracle's exact-model quotient.  The quotient amplifies root round-off
   about 1/(2h) = 100-fold, so the differences are noisy; their own noise is
   measured as the distance between steps 1e-4 and 4e-4, and the adjoint
   must be within 3x that (+1e-6) and within 1e-4.
3. The group fallback (surfdisp96 uses c0 when the second search at t1b
   finds no root, so U = c0): planted by zeroing roots at t1b, the kernels
   of those entries are the phase adjoint at t1a (within 1e-10 of the
   column's largest value: the phase sweep stops at its depth cut, the
   group sweep passes the whole stack), and every other entry is unchanged
   bit for bit."""
import numpy as np
import pytest

from conftest import rel_l2
from dazi_current_release_b200 import synthetic as S
from host_emu import emu


def _col(a, sen_off, c, K, nz):
    return a[sen_off[c]:sen_off[c + 1]].reshape((K, nz), order="F")


def _column(b, c):
    n0, n1 = b.node_off[c], b.node_off[c + 1]
    p0, p1 = b.per_off[c], b.per_off[c + 1]
    vel = np.asfortranarray(b.vs[n0:n1].reshape(1, 1, n1 - n0))
    return vel, b.depz[n0:n1], b.periods[p0:p1], p1 - p0, n1 - n0


def _run(b, ifunc, group, drop_every=0, periods=None):
    return emu.adjoint_batch(b.node_off, b.depz, b.vs, b.per_off,
                             b.periods if periods is None else periods, b.minthk, ifunc=ifunc,
                             group=group, drop_every=drop_every)


@pytest.mark.parametrize("ifunc", [2, 1])
def test_phase_adjoint_matches_exact_derivative(oracle, ifunc):
    b = S.config3(realisations=1, columns=16, base_seed=2024)
    rc, pv, st, sen, sen_off, _ = _run(b, ifunc, False)
    assert rc == 0 and (st == 0).all()
    names = ("vs", "rho") if ifunc == 1 else ("vs", "vp", "rho")
    if ifunc == 1:
        assert np.count_nonzero(sen[1]) == 0
    else:
        # the Rayleigh sweep's depth cut is exercised: pairs whose deepest
        # node, below the cut, is written as zero
        nzs = np.diff(b.node_off)
        cut = sum(int(np.count_nonzero(_col(sen[0], sen_off, c, int(b.per_off[c + 1] - b.per_off[c]),
                                            nzs[c])[:, -1] == 0.0)) for c in range(nzs.size))
        assert cut > 0
    for c in range(0, 16, 6):
        vel, depz, per, K, nz = _column(b, c)
        fine = oracle.depthkernel(vel, depz, per, b.minthk, iwave=ifunc, tol=1e-13, exact=True,
                                  dln=1e-4)
        for n in names:
            got = _col(sen[("vs", "vp", "rho").index(n)], sen_off, c, K, nz)
            err = rel_l2(got, fine["sen_" + n][0])
            assert err <= 1e-5, (c, n, err)


@pytest.mark.parametrize("ifunc", [2, 1])
def test_group_adjoint_matches_exact_derivative(oracle, ifunc):
    b = S.config3(realisations=1, columns=24, base_seed=2024)
    rc, pv, st, sen, sen_off, _ = _run(b, ifunc, True)
    assert rc == 0 and (st == 0).all()
    names = ("vs", "rho") if ifunc == 1 else ("vs", "vp", "rho")
    for c in (0, 13):
        vel, depz, per, K, nz = _column(b, c)
        kw = dict(iwave=ifunc, igr=1, tol=1e-13, exact=True)
        f1 = oracle.depthkernel(vel, depz, per, b.minthk, dln=1e-4, **kw)
        f2 = oracle.depthkernel(vel, depz, per, b.minthk, dln=4e-4, **kw)
        for n in names:
            got = _col(sen[("vs", "vp", "rho").index(n)], sen_off, c, K, nz)
            noise = rel_l2(f1["sen_" + n][0], f2["sen_" + n][0])
            err = rel_l2(got, f1["sen_" + n][0])
            assert err <= min(3.0 * noise + 1.0e-6, 1.0e-4), (c, n, err, noise)


@pytest.mark.parametrize("ifunc", [2, 1])
def test_group_fallback_is_the_phase_adjoint_at_t1a(ifunc):
    b = S.config3(realisations=1, columns=40, base_seed=99)
    rc, pv, st, full, sen_off, none = _run(b, ifunc, True)
    assert rc == 0 and not none.any()
    rc, pv2, st2, planted, _, dropped = _run(b, ifunc, True, drop_every=3)
    assert rc == 0 and dropped.sum() > 0.2 * dropped.size
    np.testing.assert_array_equal(pv2, pv)          # U itself is the reference's, untouched
    # t1a = t/(1.+h) as real*4 (surfdisp96.f:226-233): the phase adjoint there
    t1a = (b.periods / np.float64(np.float32(1.0) + np.float32(0.005))).astype(np.float32)
    rc, _, _, phase, _, _ = _run(b, ifunc, False, periods=t1a.astype(np.float64))
    assert rc == 0
    nz = np.diff(b.node_off)
    for c in range(nz.size):
        K = int(b.per_off[c + 1] - b.per_off[c])
        drop = dropped[b.per_off[c]:b.per_off[c + 1]]
        for q in range(3):
            got = _col(planted[q], sen_off, c, K, nz[c])
            # the phase adjoint sweeps to its depth cut (adj_cut_layers) and
            # the group passes the whole stack: the cut's own share is of
            # relative order exp(-32), and the two sweeps, started at
            # different depths, round differently (a few 1e-12 relative)
            ref = _col(phase[q], sen_off, c, K, nz[c])[drop]
            tol = 1.0e-10 * np.abs(ref).max(axis=-1, keepdims=True)
            np.testing.assert_allclose(got[drop], ref, rtol=0, atol=tol.max() if tol.size else 0)
            np.testing.assert_array_equal(got[~drop], _col(full[q], sen_off, c, K, nz[c])[~drop])
