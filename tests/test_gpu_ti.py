"""Gc/Gs kernel (Lsen_Gsc) on the GPU against the CPU oracle of tregn96 /
depthkernelTI.  The reference's TI A/B gate accepts rel-L2 <= 1e-5 and
max-abs <= 1e-4 for lsen_gsc (code/depthkernel_lab/run_ti_depthkernel_ab.py
:297-303); the test holds each column to that rel-L2."""
import numpy as np
import pytest

from conftest import rel_l2
import dazi_current_release_b200 as dk
from dazi_current_release_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: S.subgrid(S.config0(), 4, 3),
                                  lambda: S.subgrid(S.config1(), 4, 3),
                                  lambda: S.subgrid(S.config4(), 3, 2)])
def test_lsen_matches_oracle(oracle, make):
    case = make()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    pv, lsen = dk.depthkernelTI(nx, ny, nz, case.vel, 2, 0, K, case.periods, case.depz,
                                case.minthk, vp=case.vp, rho=case.rho)
    ref = oracle.depthkernel_ti(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                                rho=case.rho)
    np.testing.assert_array_equal(pv, ref["pvRc"])
    worst = max(rel_l2(lsen[c], ref["Lsen_Gsc"][c]) for c in range(nx * ny))
    mx = float(np.abs(lsen - ref["Lsen_Gsc"]).max())
    print(case.name, "Lsen worst per-column rel-L2", worst, "max abs", mx)
    assert worst <= 1e-5 and mx <= 1e-4


@pytest.mark.parametrize("form", [dk.FORM_PLAIN, dk.FORM_ADJOINT])
def test_fused_matches_separate_calls(form):
    case = S.subgrid(S.config1(), 3, 3)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    pv, svs, svp, srh, lsen = dk.depthkernel_fused(nx, ny, nz, case.vel, 2, 0, K, case.periods,
                                                   case.depz, case.minthk, form=form)
    pv2, svs2, svp2, srh2 = dk.depthkernel(nx, ny, nz, case.vel, 2, 0, K, case.periods, case.depz,
                                           case.minthk, form=form)
    pv3, lsen3 = dk.depthkernelTI(nx, ny, nz, case.vel, 2, 0, K, case.periods, case.depz,
                                  case.minthk)
    np.testing.assert_array_equal(pv, pv2)
    np.testing.assert_array_equal(pv, pv3)
    np.testing.assert_array_equal(svs, svs2)
    np.testing.assert_array_equal(lsen, lsen3)
