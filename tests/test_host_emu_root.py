"""The library's root search (root_kernel and its state machine), compiled
for the host by tests/host_emu, against the oracle of surfdisp96 on the CPU,
and its FP32 coarse scan (FP32 sign of the secular function on the getsol
scan steps, FP64 re-evaluation below the trust threshold and at both ends
of every bracket) against the all-FP64 scan: identical roots and statuses,
bit for bit."""
import numpy as np

from dazi_current_release_b200 import synthetic as S
from edge_models import _batch, _random_columns
from host_emu import emu


def _cases():
    b = S.config3(realisations=1, columns=240, base_seed=1000)
    yield "uneven", (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    yield "random", (*_batch(_random_columns(120, seed=3)), 2.0)


def test_fp32_scan_gives_the_fp64_roots():
    for name, args in _cases():
        rc64, pv64, st64, _ = emu.root_batch(*args, scan32=False)
        rc32, pv32, st32, _ = emu.root_batch(*args, scan32=True)
        assert rc64 == 0 and rc32 == 0
        np.testing.assert_array_equal(pv32, pv64, err_msg=name)
        np.testing.assert_array_equal(st32, st64, err_msg=name)


def test_root_search_matches_oracle_on_uneven_columns(oracle):
    b = S.config3(realisations=1, columns=240, base_seed=1000)
    rc, pv, st, _ = emu.root_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    ref = oracle.batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                       kernels=False, lsen=True)
    assert rc == 0
    np.testing.assert_array_equal(pv[:ref["pv"].size], ref["pv"])


def _tight_roots(oracle, b):
    """Per column: the reference's real*4 model, roots converged to 1e-13
    and rounded to float32 (the exact roots the Brent refinement targets)."""
    out = np.zeros(int(b.per_off[-1]))
    st = np.zeros(b.ncol, np.int32)
    for c in range(b.ncol):
        d, v, p = b.column(c)
        vp, rho = oracle.brocher(v)
        thk, rvp, rvs, rr, _ = oracle.refine(b.minthk, d, vp, v, rho)
        cg, st[c], _ = oracle.surfdisp96(thk, rvp, rvs, rr, p, tol=1e-13)
        out[b.per_off[c]:b.per_off[c + 1]] = cg
    return out, st


def test_fast_root_keeps_the_mode_and_finds_the_exact_root(oracle):
    """DAZI_FORM_FAST_ROOT: the reference's getsol scan (same bracket, same
    mode), Brent's method to 1e-10 c instead of nevill() to 1e-6 c.  Against
    the reference search: the same statuses, roots within its 1e-6 c
    tolerance (plus the two float32 roundings); against the oracle's roots
    converged to 1e-13: within one float32 ulp; and fewer evaluations."""
    b = S.config3(realisations=1, columns=240, base_seed=1000)
    args = (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    rc0, pv0, st0, ev0 = emu.root_batch(*args, scan32=False)
    rc1, pv1, st1, ev1 = emu.root_batch(*args, scan32=False, fast=True)
    assert rc0 == 0 and rc1 == 0
    np.testing.assert_array_equal(st1, st0)
    ok = pv0 > 0
    np.testing.assert_array_equal(pv1 > 0, ok)
    assert (np.abs(pv1[ok] / pv0[ok] - 1.0) <= 1e-6 + 1.3e-7).all()
    tight, st_t = _tight_roots(oracle, b)
    np.testing.assert_array_equal(st1[:b.ncol], st_t)
    ulp = np.spacing(tight[ok].astype(np.float32)).astype(np.float64)
    assert (np.abs(pv1[ok] - tight[ok]) <= ulp).all()
    print("evaluations: reference", ev0, "Brent", ev1)
    assert ev1 < 0.85 * ev0
    # with the FP32 scan the bracket is the same: the same roots
    rc2, pv2, st2, _ = emu.root_batch(*args, scan32=True, fast=True)
    np.testing.assert_array_equal(pv2, pv1)
    np.testing.assert_array_equal(st2, st1)


def test_fast_root_adjoint_kernels(oracle):
    """The adjoint form on the Brent roots: kernels within 1e-5 per column
    of the adjoint form on the reference's roots (which differ by at most
    the reference's 1e-6 c tolerance) and of the oracle's exact
    differences."""
    b = S.config3(realisations=1, columns=64, base_seed=1007)
    args = (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    r0 = emu.adjoint_batch(*args)
    r1 = emu.adjoint_batch(*args, fast=True)
    assert r0[0] == 0 and r1[0] == 0
    exact = oracle.batch_fd(*args, exact=True)
    K = np.diff(b.per_off)
    nz = np.diff(b.node_off)
    off = r1[4]
    worst_ref, worst_ex = 0.0, 0.0
    for c in range(b.ncol):
        if r1[2][c]:
            continue
        for i in range(3):
            g = r1[3][i][off[c]:off[c + 1]]
            r = r0[3][i][off[c]:off[c + 1]]
            e = exact[("sen_vs", "sen_vp", "sen_rho")[i]][off[c]:off[c + 1]]
            worst_ref = max(worst_ref, np.linalg.norm(g - r) / np.linalg.norm(r))
            worst_ex = max(worst_ex, np.linalg.norm(g - e) / np.linalg.norm(e))
    print("Brent-root adjoint vs reference-root adjoint", worst_ref, "vs exact", worst_ex)
    assert worst_ref <= 1e-5 and worst_ex <= 1e-5
    assert K.size == nz.size
