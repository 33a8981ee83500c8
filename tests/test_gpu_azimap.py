"""Azimuthal phase-velocity maps on the GPU against the oracle of
FwdAzimuthalAniMap.f90:43-86 (config-4 recipe: 2-6 % anisotropy, one fast
direction): the real*4 sums and amplitudes bit for bit, the angle to the
ulps of atan2f."""
import numpy as np
import pytest

from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.azimuthal import azimuthal_map

pytestmark = pytest.mark.gpu


def test_azimuthal_map_matches_oracle(oracle):
    case = S.subgrid(S.config4(), 5, 4)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    ti = oracle.depthkernel_ti(case.vel, case.depz, case.periods, case.minthk)
    rng = np.random.default_rng(6)
    amp = rng.uniform(0.02, 0.06, (nx - 2, ny - 2, nz - 1))
    phi = rng.uniform(0.0, np.pi, (nx - 2, ny - 2, 1))
    gc = np.asfortranarray((amp * np.cos(2 * phi)).astype(np.float32))
    gs = np.asfortranarray((amp * np.sin(2 * phi)).astype(np.float32))
    inner = [(jj * nx + ii) for jj in range(1, ny - 1) for ii in range(1, nx - 1)]
    ciso = np.asfortranarray(ti["pvRc"][inner])
    got = azimuthal_map(ti["Lsen_Gsc"], gc, gs, ciso)
    exp = oracle.azimap(ti["Lsen_Gsc"], gc, gs, ciso)
    for name, g, e in zip(("cos", "sin", "amp", "amp_rel"), got[:4], exp[:4]):
        np.testing.assert_array_equal(g, e, err_msg=name)
    d = np.abs(got[4] - exp[4])
    d = np.minimum(d, 180.0 - d)                      # angles are modulo 180 degrees
    print("angle max |diff| (deg)", d.max())
    assert d.max() <= 1e-4
