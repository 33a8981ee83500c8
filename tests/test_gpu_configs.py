"""Accuracy at every configuration's stated size (GPU against the oracle).

Each test runs the library on the whole workload of one configuration and
checks its results against the oracle: phase velocities on every column (the
oracle's phase-only path is cheap), kernels on seeded samples of columns
(the oracle's 1 + 6 nz root searches per column are not):

- config 1, 60 x 50 columns x 25 periods, plain form: all 75,000 phase
  velocities bit-identical to the oracle's (float32 rounding-midpoint flips
  excepted), FD kernels on 300 columns as the oracle's;
- config 2, 100 x 100 x 30, adjoint form: kernels on 200 columns within
  1e-4 rel-L2 of the oracle's exact differences (the north star's bound);
- config 4, 200 x 200 x 40: FP32 scan and all-FP64 scan give the same
  1.6 M phase velocities; 200 columns against the oracle; the Brent
  refinement within the reference's tolerance;
- config 3, 1,000 columns drawn from the 250,000 of the uneven batch:
  status (first period without a root) and fundamental-mode identity per
  column, default and Brent refinement; Lsen_Gsc on 100 of them.
"""
import numpy as np
import pytest

from conftest import assert_fd_parity, assert_pv_parity, rel_l2
import dazi_current_release_b200 as dk
from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.batch import depthkernel_batch
from dazi_current_release_b200.depthkernel import last_status

pytestmark = pytest.mark.gpu


def _columns(case, idx):
    """The grid columns idx as an (n, 1, nz) grid (Fortran order)."""
    nx, ny, nz = case.vel.shape
    flat = case.vel.reshape(nx * ny, nz, order="F")
    return np.asfortranarray(flat[idx].reshape(len(idx), 1, nz))


def _grid_pv_oracle(oracle, case):
    r = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, kernels=False)
    d = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, kernels=False,
                           round_f32=False)
    return r["pvRc"], d["pvRc"], r["status"]


def test_config1_full_grid_plain_form(oracle):
    case = S.config1()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    pv, svs, svp, srh = dk.depthkernel(nx, ny, nz, case.vel, 2, 0, K, case.periods, case.depz,
                                       case.minthk, form=dk.FORM_PLAIN)
    st = last_status(nx * ny)
    ref, ref_d, ref_st = _grid_pv_oracle(oracle, case)
    np.testing.assert_array_equal(st, ref_st)
    flips = assert_pv_parity(pv.ravel(), ref.ravel(), ref_d.ravel(), allow_tol_moves=True)
    assert flips <= max(2, pv.size // 1000), flips
    idx = np.sort(np.random.default_rng(11).choice(nx * ny, 300, replace=False))
    sub = _columns(case, idx)
    refk = oracle.depthkernel(sub, case.depz, case.periods, case.minthk)
    vp, rho = oracle.brocher(sub.reshape(-1))
    vp, rho = vp.reshape(len(idx), nz), rho.reshape(len(idx), nz)
    worst, differ = 0.0, 0
    for j, c in enumerate(idx):
        for got, exp, x in ((svs[c], refk["sen_vs"][j], sub[j, 0]), (svp[c], refk["sen_vp"][j], vp[j]),
                            (srh[c], refk["sen_rho"][j], rho[j])):
            worst = max(worst, rel_l2(got, exp))
            differ += assert_fd_parity(got, exp, x)
    print(f"config 1: pv flips {flips} of {pv.size}; kernels on 300 columns worst rel-L2 "
          f"{worst:.2e}, {differ} of {3 * 300 * K * nz} entries differ")
    assert worst <= 1e-4


def test_config2_adjoint_form_against_exact_differences(oracle):
    case = S.config2()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    pv, svs, svp, srh = dk.depthkernel(nx, ny, nz, case.vel, 2, 0, K, case.periods, case.depz,
                                       case.minthk, form=dk.FORM_ADJOINT)
    idx = np.sort(np.random.default_rng(12).choice(nx * ny, 200, replace=False))
    sub = _columns(case, idx)
    ex = oracle.depthkernel(sub, case.depz, case.periods, case.minthk, exact=True, tol=1e-13,
                            dln=1e-4)
    ref = oracle.depthkernel(sub, case.depz, case.periods, case.minthk, kernels=False)
    ref_d = oracle.depthkernel(sub, case.depz, case.periods, case.minthk, kernels=False,
                               round_f32=False)
    flips = assert_pv_parity(pv[idx].ravel(), ref["pvRc"].ravel(), ref_d["pvRc"].ravel(),
                             allow_tol_moves=True)
    assert flips <= max(2, ref["pvRc"].size // 1000), flips
    worst = {"sen_vs": 0.0, "sen_vp": 0.0, "sen_rho": 0.0}
    for j, c in enumerate(idx):
        for name, got in (("sen_vs", svs), ("sen_vp", svp), ("sen_rho", srh)):
            worst[name] = max(worst[name], rel_l2(got[c], ex[name][j]))
    print("config 2: adjoint kernels vs exact differences, worst per-column rel-L2", worst)
    assert max(worst.values()) <= 1e-4


def test_config4_fp32_scan_fp64_scan_and_oracle(oracle):
    case = S.config4()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    run = lambda form: dk.depthkernel(nx, ny, nz, case.vel, 2, 0, K, case.periods,  # noqa: E731
                                      case.depz, case.minthk, form=form, kernels=False)[0]
    pv64 = run(dk.FORM_ADJOINT)
    st64 = last_status(nx * ny)
    pv32 = run(dk.FORM_ADJOINT | dk.FORM_SCAN_FP32)
    st32 = last_status(nx * ny)
    np.testing.assert_array_equal(pv32, pv64)
    np.testing.assert_array_equal(st32, st64)
    pvf = run(dk.FORM_ADJOINT | dk.FORM_FAST_ROOT)
    np.testing.assert_array_equal(last_status(nx * ny), st64)
    ok = pv64 > 0
    fast_rel = float(np.abs(pvf[ok] / pv64[ok] - 1.0).max())
    assert fast_rel <= 1e-6 + 1.3e-7
    idx = np.sort(np.random.default_rng(13).choice(nx * ny, 200, replace=False))
    sub = _columns(case, idx)
    ref = oracle.depthkernel(sub, case.depz, case.periods, case.minthk, kernels=False)
    ref_d = oracle.depthkernel(sub, case.depz, case.periods, case.minthk, kernels=False,
                               round_f32=False)
    flips = assert_pv_parity(pv64[idx].ravel(), ref["pvRc"].ravel(), ref_d["pvRc"].ravel(),
                             allow_tol_moves=True)
    assert flips <= max(2, ref["pvRc"].size // 1000), flips
    np.testing.assert_array_equal(st64[idx], ref["status"])
    print(f"config 4: {pv64.size} phase velocities, FP32 scan = FP64 scan; 200 columns vs "
          f"oracle: {flips} midpoint flips; Brent refinement max rel diff {fast_rel:.2e}")


def test_config3_status_and_mode_identity(oracle):
    full = S.config3()
    idx = np.sort(np.random.default_rng(14).choice(full.ncol, 1000, replace=False))
    nz = np.diff(full.node_off)[idx]
    K = np.diff(full.per_off)[idx]
    cat = lambda arr, off: np.concatenate([arr[off[c]:off[c + 1]] for c in idx])  # noqa: E731
    b = S.RaggedBatch(np.concatenate([[0], np.cumsum(nz)]).astype(np.int64),
                      cat(full.depz, full.node_off), cat(full.vs, full.node_off),
                      np.concatenate([[0], np.cumsum(K)]).astype(np.int64),
                      cat(full.periods, full.per_off), full.minthk)
    args = (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    ref = oracle.batch(*args, kernels=False, lsen=False)
    st_ref = np.array([next((k + 1 for k, v in enumerate(ref["pv"][b.per_off[c]:b.per_off[c + 1]])
                             if v == 0), 0) for c in range(b.ncol)], np.int32)
    r0 = depthkernel_batch(*args, form=dk.FORM_ADJOINT, kernels=False, lsen=False)
    r1 = depthkernel_batch(*args, form=dk.FORM_ADJOINT | dk.FORM_FAST_ROOT, kernels=False,
                           lsen=False)
    np.testing.assert_array_equal(r0["status"], st_ref)
    np.testing.assert_array_equal(r1["status"], st_ref)
    ok = ref["pv"] > 0
    # default search: the reference's points, the reference's roots
    differ = int(np.count_nonzero(r0["pv"] != ref["pv"]))
    assert (np.abs(r0["pv"][ok] / ref["pv"][ok] - 1.0) <= 1e-6).all()
    assert differ <= max(2, b.column_periods // 1000), differ
    # Brent refinement: the same bracket, the root within the reference's tolerance
    assert (np.abs(r1["pv"][ok] / ref["pv"][ok] - 1.0) <= 1e-6 + 1.3e-7).all()
    # Lsen_Gsc on 100 of the columns (the TI oracle at its real*4 roots)
    sub = np.arange(0, b.ncol, 10)
    nzs, Ks = nz[sub], K[sub]
    bb = S.RaggedBatch(np.concatenate([[0], np.cumsum(nzs)]).astype(np.int64),
                       np.concatenate([b.column(int(c))[0] for c in sub]),
                       np.concatenate([b.column(int(c))[1] for c in sub]),
                       np.concatenate([[0], np.cumsum(Ks)]).astype(np.int64),
                       np.concatenate([b.column(int(c))[2] for c in sub]), b.minthk)
    a2 = (bb.node_off, bb.depz, bb.vs, bb.per_off, bb.periods, bb.minthk)
    rl = depthkernel_batch(*a2, form=dk.FORM_ADJOINT, kernels=False, lsen=True)
    rol = oracle.batch(*a2, kernels=False, lsen=True)
    worst = 0.0
    for c in range(bb.ncol):
        lo, hi = rol["ls_off"][c], rol["ls_off"][c + 1]
        assert (rl["ls_off"][c], rl["ls_off"][c + 1]) == (lo, hi)
        worst = max(worst, rel_l2(rl["lsen"][lo:hi], rol["lsen"][lo:hi]))
    print(f"config 3: 1000 columns, {int(ok.sum())} roots; statuses equal; default search "
          f"{differ} values differ (midpoint flips / root-tolerance moves); Lsen worst "
          f"per-column rel-L2 {worst:.2e} on 100 columns")
    assert worst <= 1e-5
