"""The CPU oracle against the reference's own golden output.

examples/test4_Yunnan/*/period_phaseVMOD.dat is the Fortran surfdisp96 phase
velocity of the inner columns of the Yunnan initial model (f10.4 print).
The oracle must reproduce the legacy-parameter run exactly after the same
rounding, and the current run within one print step (the two reference runs
themselves differ by one step in 49 rows)."""
import numpy as np
import pytest

from conftest import inner_columns


def _oracle_pv(oracle, y):
    r = oracle.depthkernel(y["vel"], y["depz"], y["periods"], float(y["minthk"]), kernels=False)
    assert (r["status"] == 0).all()
    return r


def test_oracle_matches_legacy_golden_exactly(oracle, yunnan):
    r = _oracle_pv(oracle, yunnan)
    mine = inner_columns(r["pvRc"], int(yunnan["nx"]), int(yunnan["ny"]))
    printed = np.rint(mine * 1e4).astype(np.int64)
    gold = yunnan["pv_legacy_e4"].astype(np.int64)
    assert printed.shape == gold.shape
    assert np.array_equal(printed, gold)


def test_oracle_within_one_print_step_of_current_golden(oracle, yunnan):
    r = _oracle_pv(oracle, yunnan)
    mine = inner_columns(r["pvRc"], int(yunnan["nx"]), int(yunnan["ny"]))
    gold = yunnan["pv_current_e4"].astype(np.float64) * 1e-4
    assert np.abs(mine - gold).max() <= 0.5e-4 + 2e-6
    diff_rows = np.count_nonzero(np.rint(mine * 1e4) != yunnan["pv_current_e4"])
    assert diff_rows <= 0.001 * gold.size


def test_refinement_layer_counts(oracle, yunnan):
    vs = np.full(21, 3.5, np.float32)
    vp, rho = oracle.brocher(vs)
    out = oracle.refine(4.0, (3.0 * np.arange(21)).astype(np.float32), vp, vs, rho)
    assert out[0].size == 101                       # 20 intervals x 5 + half-space
    assert out[0][-1] == 0.0 and (out[4] == 5).all()
    vs = np.full(18, 3.5, np.float32)
    vp, rho = oracle.brocher(vs)
    out = oracle.refine(4.0, yunnan["depz"], vp, vs, rho)
    assert out[0].size == 86                        # Yunnan grid, rmax = 86


def test_halfspace_rayleigh_speed(oracle):
    """Uniform Poisson solid: flat-earth phase velocity is 0.9194 Vs."""
    vs = np.float32(3.5)
    vp = np.float32(vs * np.sqrt(3.0))
    thk = np.array([5.0] * 10 + [0.0], np.float32)
    cg, st, ev = oracle.surfdisp96(thk, np.full(11, vp), np.full(11, vs), np.full(11, 2.7, np.float32),
                                   np.array([5.0, 10.0]), iflsph=0)
    assert st == 0
    np.testing.assert_allclose(cg, 0.919402 * 3.5, rtol=2e-6)


def test_no_root_zero_fills_remaining_periods(oracle):
    """surfdisp96.f:1700-1770: no root -> this and later periods are zero."""
    thk = np.array([2.0, 0.0], np.float32)
    vs = np.array([3.0, 3.0], np.float32)
    vp = np.array([5.2, 5.2], np.float32)
    rho = np.array([2.7, 2.7], np.float32)
    # tolerance 0 keeps nevill iterating; a degenerate period list with a
    # non-positive period has no root at all
    cg, st, ev = oracle.surfdisp96(thk, vp, vs, rho, np.array([5.0, -1.0, 10.0]))
    assert st == 2 and cg[0] > 0 and cg[1] == 0 and cg[2] == 0


@pytest.mark.parametrize("tol", [1e-6, 1e-10])
def test_tolerance_knob_changes_root_at_most_tol(oracle, tol):
    from dazi_current_release_b200 import synthetic as S
    case = S.subgrid(S.config1(), 3, 2)
    ref = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, kernels=False,
                             tol=1e-13, round_f32=False)["pvRc"]
    got = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, kernels=False,
                             tol=tol, round_f32=False)["pvRc"]
    assert np.abs(got / ref - 1).max() <= 1.01 * tol
