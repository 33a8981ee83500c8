"""The CPU oracle of tregn96 / depthkernelTI, checked by physics.

No golden vector of the reference pins Lsen_Gsc.  With sphericity and Q
switched off, tregn96's variational partials of an isotropic layered model
must equal derivatives of the surfdisp96 root: dc/dVs(layer) = dcdbv + dcdbh
(dcdbh = 0 for Rayleigh waves), dc/dVp(layer) = dcdah + dcdav, and the
phase velocity is invariant under a density scaling at fixed velocities."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def flat_model():
    thk = np.array([2.0] * 20 + [0.0])
    vs = np.linspace(2.8, 4.5, 21)
    vp = 1.75 * vs
    rho = 2.0 + 0.3 * vs
    per = np.array([5.0, 10.0, 20.0, 40.0])
    return thk, vp, vs, rho, per


def _ti_inputs(vp, vs, rho):
    f32 = lambda x: np.asarray(x, np.float32)  # noqa: E731
    TA = f32(rho) * f32(vp) ** 2
    TL = f32(rho) * f32(vs) ** 2
    return TA, TA, TA - 2 * TL, TL, TL


def _fd(oracle, thk, vp, vs, rho, per, which, h=1e-5):
    out = []
    for m in range(len(thk)):
        arrs = [thk, vp.copy(), vs.copy(), rho.copy()]
        arrs[which][m] += h
        cp, _ = oracle.surfdisp96_d(*arrs, per, iflsph=0)
        arrs[which][m] -= 2 * h
        cm, _ = oracle.surfdisp96_d(*arrs, per, iflsph=0)
        out.append((cp - cm) / (2 * h))
    return np.array(out).T


def test_tregn96_partials_equal_root_derivatives(oracle, flat_model):
    thk, vp, vs, rho, per = flat_model
    c, st = oracle.surfdisp96_d(thk, vp, vs, rho, per, iflsph=0)
    assert st == 0
    TA, TC, TF, TL, TN = _ti_inputs(vp, vs, rho)
    *_, full = oracle.tregn96(thk, TA, TC, TF, TL, TN, rho, per, c, nsph=0, dogam=0, full=True)
    fd_b = _fd(oracle, thk, vp, vs, rho, per, 2)
    fd_a = _fd(oracle, thk, vp, vs, rho, per, 1)
    for k in range(per.size):
        eb = np.linalg.norm(full[k][3] + full[k][2] - fd_b[k]) / np.linalg.norm(fd_b[k])
        ea = np.linalg.norm(full[k][0] + full[k][1] - fd_a[k]) / np.linalg.norm(fd_a[k])
        assert eb < 2e-6 and ea < 1e-5, (per[k], eb, ea)
        rho32 = np.asarray(rho, np.float32).astype(np.float64)
        assert abs((rho32 * full[k][5]).sum()) < 1e-6 * c[k]


def test_q_shift_and_sphericity_are_small_and_signed(oracle, flat_model):
    """dogam: attenuation lowers c at periods above 1 s (log(omega/2pi) < 0);
    the shift is a fraction of a percent for Q = 150/50."""
    thk, vp, vs, rho, per = flat_model
    c, _ = oracle.surfdisp96_d(thk, vp, vs, rho, per, iflsph=0)
    TA, TC, TF, TL, TN = _ti_inputs(vp, vs, rho)
    *_, full = oracle.tregn96(thk, TA, TC, TF, TL, TN, rho, per, c, nsph=0, dogam=1, full=True)
    cq = full[:, 6, 0]
    rel = cq / c - 1
    assert (rel < 0).all() and (rel > -0.05).all()


def test_depthkernel_ti_runs_config0(oracle):
    from dazi_current_release_b200 import synthetic as S
    case = S.subgrid(S.config0(), 3, 2)
    r = oracle.depthkernel_ti(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                              rho=case.rho)
    L = r["Lsen_Gsc"]
    assert L.shape == (6, case.periods.size, case.depz.size - 1)
    assert np.isfinite(L).all() and (np.abs(L).sum(axis=2) > 0).all()
    # pv equals the iso oracle's
    iso = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                             rho=case.rho, kernels=False)
    np.testing.assert_array_equal(r["pvRc"], iso["pvRc"])
