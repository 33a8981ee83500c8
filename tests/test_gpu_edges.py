"""Edge cases of the stage on the GPU, through the ragged batch C-ABI, against
the CPU oracle: columns without a fundamental-mode root (the reference
zero-fills that period and every later one, surfdisp96.f:1700-1770), the
compiled maximum sizes (nz <= 200 nodes, kmaxRc <= 160 periods, <= 200
refined layers, surfdisp96.f:57-59) and the limits beyond them, the
smallest column (one layer over the half-space, one period) and an empty
batch."""
import ctypes

import numpy as np
import pytest

from conftest import assert_fd_parity, assert_pv_parity, rel_l2
from edge_models import _batch, _random_columns, leaky_periods
import dazi_current_release_b200 as dk
from dazi_current_release_b200 import _lib
from dazi_current_release_b200.batch import depthkernel_batch

pytestmark = pytest.mark.gpu


def _check_against_oracle(oracle, cols, minthk, r, kernels=True):
    node_off, depz, vs, per_off, per = _batch(cols)
    ref = oracle.batch(node_off, depz, vs, per_off, per, minthk, kernels=kernels)
    failed = 0
    fd_diff = fd_total = 0
    leaky = [0]
    pv_diff = pv_total = 0
    for c, (dep, v, p) in enumerate(cols):
        a, b = per_off[c], per_off[c + 1]
        pv_ref = ref["pv"][a:b]
        nroot = int(np.argmin(pv_ref > 0)) if (pv_ref <= 0).any() else p.size
        # status: first period without a root (1-based), 0 if none
        assert r["status"][c] == (0 if nroot == p.size else nroot + 1), c
        failed += nroot < p.size
        unr = oracle.depthkernel(v.reshape(1, 1, -1), dep, p, minthk, round_f32=False,
                                 kernels=False)["pvRc"][0]
        got = r.column(c)
        pv_diff += assert_pv_parity(got[0], pv_ref, unr, allow_tol_moves=True)
        pv_total += p.size
        K, nz = p.size, dep.size
        q = 1
        if kernels:
            # plain form: the reference's central differences at every
            # period, also past a failed one (its perturbed models may
            # still have roots, DepthKernel1D.f90:141-181)
            s0, s1 = ref["sen_off"][c], ref["sen_off"][c + 1]
            vp, rho = oracle.brocher(v)
            for name, x in (("sen_vs", v), ("sen_vp", vp), ("sen_rho", rho)):
                exp = ref[name][s0:s1].reshape((K, nz), order="F")
                g = got[q]
                q += 1
                fd_diff += assert_fd_parity(g, exp, x, max_frac=1.0)
                fd_total += g.size
        l0, l1 = ref["ls_off"][c], ref["ls_off"][c + 1]
        exp = ref["lsen"][l0:l1].reshape((K, nz - 1), order="F")
        g = got[-1]
        assert (g[nroot:] == 0).all()
        assert np.isfinite(g).all()
        # not comparable above the half-space's P speed (leaky_periods)
        # and Lsen is compared where its input, the phase velocity, is the
        # oracle's bit for bit (a root that moved within its tolerance can
        # move Lsen by more near the half-space's S speed)
        ok = np.nonzero(~leaky_periods(pv_ref[:nroot], v[-1], oracle.brocher)
                        & (got[0][:nroot] == pv_ref[:nroot]))[0]
        leaky[0] += nroot - ok.size
        if ok.size:
            assert rel_l2(g[ok], exp[ok]) <= 1e-5, c
            assert np.abs(g[ok] - exp[ok]).max() <= 1e-4, c
    # differing FD entries (each within the root tolerance, checked above):
    # a small share, from roots of these high-contrast models that moved
    # within the tolerance and carried the move to the later periods
    print("FD entries differing within the root tolerance:", fd_diff, "of", fd_total)
    assert fd_diff <= max(3, 0.05 * fd_total), (fd_diff, fd_total)
    print("periods above the half-space P speed (Lsen not compared):", leaky[0])
    print("phase velocities differing (rounding flips / moves within 1e-6 c):", pv_diff,
          "of", pv_total)
    assert pv_diff <= max(2, 0.02 * pv_total)
    return failed


def test_columns_without_a_root_match_oracle(oracle):
    cols = _random_columns(60)
    node_off, depz, vs, per_off, per = _batch(cols)
    r = depthkernel_batch(node_off, depz, vs, per_off, per, 2.0, form=dk.FORM_PLAIN)
    failed = _check_against_oracle(oracle, cols, 2.0, r)
    print("columns with a failed period:", failed)
    assert failed >= 3
    # the adjoint form reports the same roots and statuses; its kernels are
    # zero from the first failed period on (no root, no derivative)
    ra = depthkernel_batch(node_off, depz, vs, per_off, per, 2.0, form=dk.FORM_ADJOINT)
    np.testing.assert_array_equal(ra["pv"], r["pv"])
    np.testing.assert_array_equal(ra["status"], r["status"])
    np.testing.assert_array_equal(ra["lsen"], r["lsen"])
    for c in range(len(cols)):
        if ra["status"][c]:
            for g in ra.column(c)[1:4]:
                assert (g[ra["status"][c] - 1:] == 0).all()


def _max_column(seed, nz=200, K=160):
    rng = np.random.default_rng(seed)
    dep = np.concatenate([[0.0], np.cumsum(rng.uniform(0.3, 1.2, nz - 1))]).astype(np.float32)
    vs = ((2.6 + 2.0 * dep / dep[-1]) * (1.0 + 0.03 * rng.standard_normal(nz))).astype(np.float32)
    per = np.geomspace(2.0, 100.0, K)
    return dep, vs, per


def test_maximum_sizes_match_oracle(oracle):
    # minthk 0.5 gives one sublayer per layer: 199 layers + half-space = 200
    cols = [_max_column(11), _max_column(12)]
    node_off, depz, vs, per_off, per = _batch(cols)
    r = depthkernel_batch(node_off, depz, vs, per_off, per, 0.5, form=dk.FORM_ADJOINT)
    _check_against_oracle(oracle, cols, 0.5, r, kernels=False)
    assert (r["status"] == 0).all()


def _raw_batch(cols, minthk, form=dk.FORM_ADJOINT):
    L = _lib.load()
    node_off, depz, vs, per_off, per = _batch(cols)
    n = len(cols)
    K = np.diff(per_off)
    nz = np.diff(node_off)
    sen_off = np.concatenate([[0], np.cumsum(K * nz)]).astype(np.int64)
    ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))]).astype(np.int64)
    pv = np.zeros(max(int(per_off[-1]), 1))
    sen = [np.zeros(max(int(sen_off[-1]), 1)) for _ in range(3)]
    ls = np.zeros(max(int(ls_off[-1]), 1), np.float32)
    st = np.zeros(max(n, 1), np.int32)
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    i64, f32, f64 = ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    return L.dazi_dk_batch(n, P(node_off, i64), P(depz, f32), P(vs, f32), None, None,
                           P(per_off, i64), P(per, f64), ctypes.c_float(minthk), P(pv, f64),
                           P(sen_off, i64), P(sen[0], f64), P(sen[1], f64), P(sen[2], f64),
                           P(ls_off, i64), P(ls, f32), form, P(st, ctypes.c_int))


@pytest.mark.parametrize("nz,K,minthk", [(201, 10, 0.5),    # nodes beyond 200
                                         (50, 161, 0.5),    # periods beyond 160
                                         (120, 10, 1.0)])   # 239 refined layers
def test_beyond_limits_rejected(nz, K, minthk):
    col = _max_column(3, nz=nz, K=K)
    assert _raw_batch([col], minthk) == _lib.DAZI_ERR_LIMITS
    assert len(_lib.load().dazi_dk_last_error()) > 0
    # the library stays usable after the rejection
    assert _raw_batch([_max_column(4, nz=20, K=5)], 2.0) == _lib.DAZI_OK


def test_smallest_column_and_empty_batch(oracle):
    cols = [(np.array([0.0, 5.0], np.float32), np.array([3.0, 4.2], np.float32),
             np.array([8.0]))]
    node_off, depz, vs, per_off, per = _batch(cols)
    r = depthkernel_batch(node_off, depz, vs, per_off, per, 2.0, form=dk.FORM_PLAIN)
    _check_against_oracle(oracle, cols, 2.0, r)
    assert _raw_batch([], 2.0) == _lib.DAZI_OK
