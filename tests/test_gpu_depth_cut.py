"""The depth cut of the Rayleigh phase adjoint and Gc/Gs sweeps against the
same sweeps over the whole stack (DAZI_FORM_FULL_STACK), on 1,000 columns of
the uneven workload (config 3 recipe):
- the phase velocities and statuses are the same (the root search has no
  cut);
- the adjoint kernels differ by at most 1e-10 of each column's largest
  value (the stack below the cut contributes exp(-32) relative; the two
  sweeps also round differently);
- Lsen_Gsc (real*4) differs by at most 1e-7 per-column rel-L2;
- the cut is reached: some deepest nodes are zero with the cut and non-zero
  without it."""
import numpy as np
import pytest

import dazi_current_release_b200 as dk
from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.batch import depthkernel_batch

pytestmark = pytest.mark.gpu


def test_cut_against_full_stack():
    b = S.config3(realisations=1, columns=1000, base_seed=4242)
    run = lambda form: depthkernel_batch(b.node_off, b.depz, b.vs, b.per_off,  # noqa: E731
                                         b.periods, b.minthk, form=form)
    cut = run(dk.FORM_ADJOINT)
    full = run(dk.FORM_ADJOINT | dk.FORM_FULL_STACK)
    np.testing.assert_array_equal(cut["pv"], full["pv"])
    np.testing.assert_array_equal(cut["status"], full["status"])
    worst_sen, worst_ls, reached = 0.0, 0.0, 0
    for c in range(b.ncol):
        a, f = cut.column(c), full.column(c)
        for q in (1, 2, 3):          # sen_vs, sen_vp, sen_rho: (K, nz)
            scale = np.abs(f[q]).max()
            if scale > 0:
                worst_sen = max(worst_sen, float(np.abs(a[q] - f[q]).max() / scale))
        reached += int(np.count_nonzero((a[1][:, -1] == 0.0) & (f[1][:, -1] != 0.0)))
        den = np.linalg.norm(f[4])
        if den > 0:
            worst_ls = max(worst_ls, float(np.linalg.norm(a[4] - f[4]) / den))
    print(f"cut vs full stack: kernels {worst_sen:.2e} of the column maximum, "
          f"Lsen rel-L2 {worst_ls:.2e}, {reached} (column, period) pairs cut")
    assert worst_sen <= 1e-10
    assert worst_ls <= 1e-7
    assert reached > 0
