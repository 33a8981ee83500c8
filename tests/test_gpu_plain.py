"""Plain (perturb-and-recompute) GPU form against the CPU oracle and the
reference's golden phase velocities.  Calls go through the C-ABI."""
import numpy as np
import pytest

from conftest import assert_pv_parity, inner_columns, rel_l2
import dazi_current_release_b200 as dk
from dazi_current_release_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def test_gpu_pv_matches_legacy_golden_exactly(yunnan):
    y = yunnan
    nx, ny, nz = int(y["nx"]), int(y["ny"]), int(y["nz"])
    (pv,) = dk.depthkernel(nx, ny, nz, y["vel"], 2, 0, y["periods"].size, y["periods"], y["depz"],
                           float(y["minthk"]), form=dk.FORM_PLAIN, kernels=False)
    printed = np.rint(inner_columns(pv, nx, ny) * 1e4).astype(np.int64)
    assert np.array_equal(printed, y["pv_legacy_e4"].astype(np.int64))


def _plain(case, **kw):
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    if case.vp is not None:
        return dk.depthkernel_vpvsrho(nx, ny, nz, case.vel, case.vp, case.rho, 2, 0, K,
                                      case.periods, case.depz, case.minthk,
                                      form=dk.FORM_PLAIN, **kw)
    return dk.depthkernel(nx, ny, nz, case.vel, 2, 0, K, case.periods, case.depz, case.minthk,
                          form=dk.FORM_PLAIN, **kw)


def _compare(case, oracle, col_tol=1e-4):
    pv, svs, svp, srh = _plain(case)
    ref = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                             rho=case.rho)
    assert (ref["status"] == 0).all()
    # phase velocity: the oracle's sngl(c) bit for bit (up to a root that
    # sits on a float32 rounding midpoint), so within 1e-6 relative
    unr = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                             rho=case.rho, round_f32=False, kernels=False)["pvRc"]
    nxy = pv.shape[0]
    flips = sum(assert_pv_parity(pv[c], ref["pvRc"][c], unr[c]) for c in range(nxy))
    assert flips <= max(1, pv.size // 500)
    np.testing.assert_array_less(np.abs(pv / ref["pvRc"] - 1.0), 1e-6)
    worst = 0.0
    for name, got, exp in (("vs", svs, ref["sen_vs"]), ("vp", svp, ref["sen_vp"]),
                           ("rho", srh, ref["sen_rho"])):
        for c in range(nxy):
            e = rel_l2(got[c], exp[c])
            worst = max(worst, e)
            assert e <= col_tol, (name, c, e)
    return pv, worst


def test_plain_fd_matches_oracle_config0(oracle):
    case = S.config0()
    _, worst = _compare(case, oracle)
    print("config0 worst per-column rel-L2", worst)


def test_plain_fd_matches_oracle_config1_subgrid(oracle):
    case = S.subgrid(S.config1(), 6, 5)
    _, worst = _compare(case, oracle)
    print("config1 subgrid worst per-column rel-L2", worst)


def test_plain_fd_matches_oracle_config2_subgrid(oracle):
    case = S.subgrid(S.config2(), 4, 3)
    _, worst = _compare(case, oracle)
    print("config2 subgrid worst per-column rel-L2", worst)


def test_plain_fd_matches_oracle_config4_subgrid(oracle):
    case = S.subgrid(S.config4(), 3, 2)
    _, worst = _compare(case, oracle)
    print("config4 subgrid worst per-column rel-L2", worst)


def test_column_range_writes_only_that_range(oracle):
    case = S.subgrid(S.config1(), 4, 3)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    full = _plain(case)
    pv = np.full((nx * ny, K), -7.0, order="F")
    sen = tuple(np.full((nx * ny, K, nz), -7.0, order="F") for _ in range(3))
    from dazi_current_release_b200.depthkernel import _run_iso
    _run_iso(nx, ny, nz, case.vel, None, None, 2, 0, K, case.periods, case.depz, case.minthk,
             dk.FORM_PLAIN, 5, 4, True, pvRc=pv, sen=sen)
    assert (pv[:4] == -7).all() and (pv[8:] == -7).all()
    np.testing.assert_array_equal(pv[4:8], full[0][4:8])
    for a, b in zip(sen, full[1:]):
        np.testing.assert_array_equal(a[4:8], b[4:8])
        assert (a[:4] == -7).all()
