"""The library's kernels against the reference's pDSurf tile backend run
(tests/golden/pdsurf_fd.npz, made by tests/golden/make_pdsurf_fd.py), with
the reference's A/B gates widened only by pDSurf's own difference noise
(see tests/test_oracle_pdsurf.py): the plain form, and the adjoint form
(the exact derivative, so its distance to pDSurf is pDSurf's noise)."""
import numpy as np
import pytest

import dazi_current_release_b200 as dk
from test_oracle_pdsurf import GATES, check_against_pdsurf, pdsurf_case  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", [dk.FORM_PLAIN, dk.FORM_ADJOINT])
def test_kernels_match_the_reference_pdsurf_run(pdsurf_case, form):  # noqa: F811
    c = pdsurf_case
    sub = c["sub"]
    n, _, nz = sub.shape
    per = c["f"]["periods"]
    pv, svs, svp, srh = dk.depthkernel(n, 1, nz, sub, 2, 0, per.size, per, c["depz"],
                                       c["minthk"], form=form)
    out = check_against_pdsurf(dict(pvRc=pv, sen_vs=svs, sen_vp=svp, sen_rho=srh), c)
    print(form, {k: f"{v[0]:.2e}" for k, v in out.items()})
    if form == dk.FORM_ADJOINT:
        for k, (_, noise, to_exact) in out.items():
            assert to_exact <= 1e-4, (k, to_exact)
