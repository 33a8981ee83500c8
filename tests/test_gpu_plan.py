"""Plans (one CUDA-graph launch per run, kernel variants picked by the
autotuner) against the per-call batch entry: same roots and statuses bit
for bit, kernels to rounding (variants differ only in register budgets),
and a second run after the velocities change in place."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
import dazi_current_release_b200 as dk
from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.batch import depthkernel_batch
from dazi_current_release_b200.plan import BatchPlan

pytestmark = pytest.mark.gpu


def _check(plan, b, vs):
    ref = depthkernel_batch(b.node_off, b.depz, vs, b.per_off, b.periods, b.minthk,
                            form=dk.FORM_ADJOINT)
    np.testing.assert_array_equal(plan.pv.cpu().numpy(), ref["pv"])
    np.testing.assert_array_equal(plan.status.cpu().numpy(), ref["status"])
    for name in ("sen_vs", "sen_vp", "sen_rho"):
        assert rel_l2(getattr(plan, name).cpu().numpy(), ref[name]) <= 1e-12, name
    assert rel_l2(plan.lsen.cpu().numpy(), ref["lsen"]) <= 1e-6


def test_plan_matches_batch_and_reruns():
    b = S.config3(realisations=1, columns=2500, base_seed=1007)
    plan = BatchPlan(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    cfg = plan.config()
    print("autotuner:", cfg)
    assert cfg["root_block"] in (64, 128, 256)
    assert cfg["adjoint_blocks_per_sm"] in (2, 3, 4)
    assert cfg["ti_blocks_per_sm"] in (2, 3, 4, 6, 8)
    plan.run()
    torch.cuda.synchronize()
    plan.status_check()
    _check(plan, b, b.vs)
    # new velocities written into the bound buffer, same structure
    rng = np.random.default_rng(5)
    vs2 = (b.vs * (1.0 + 0.02 * rng.standard_normal(b.vs.size))).astype(np.float32)
    plan.vs.copy_(torch.as_tensor(vs2))
    plan.run()
    torch.cuda.synchronize()
    _check(plan, b, vs2)
    plan.close()


def test_plan_rejects_plain_form():
    from dazi_current_release_b200 import _lib
    import ctypes
    L = _lib.load()
    h = ctypes.c_void_p(None)
    rc = L.dazi_dk_plan_create(1, None, None, None, None, None, None, None, ctypes.c_float(2.0),
                               None, None, None, None, None, None, None, 0, None, 1, None,
                               ctypes.byref(h))
    assert rc == _lib.DAZI_ERR_BADARG
