"""Love waves and group velocity on the GPU (surfdisp96 iwave = 1, igr > 0),
through the C-ABI, against the oracle and the reference's own Python surf96.

Tolerances as in test_host_emu_wave.py: two root searches of one zero end
at most 2e-6 c apart (each stops on a bracket narrower than 1e-6 c,
surfdisp96.f:608); the group velocity's difference quotient over
t/(1 -+ h), h = 0.005, turns that into at most ~4e-4 U.  Love evaluates
dltar1 in the reference's operation order and matches bit for bit."""
import numpy as np
import pytest

from conftest import assert_fd_parity
import dazi_current_release_b200 as dk
from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.batch import depthkernel_batch

pytestmark = pytest.mark.gpu

PHASE_MOVE = 2.0e-6
GROUP_MOVE = 4.0e-4
COMBOS = [(2, 0), (2, 1), (1, 0), (1, 1)]


def _moves_ok(got, ref, iwave, igr, max_frac=0.05):
    """pv against the oracle: equal, or moved within the root tolerance."""
    got = np.asarray(got, np.float64).ravel()
    ref = np.asarray(ref, np.float64).ravel()
    moved = np.nonzero(got != ref)[0]
    if iwave == 1:
        assert moved.size <= max(1, got.size // 1000), moved[:5]
    assert moved.size <= max(2, max_frac * got.size), moved.size
    assert np.all(ref[moved] > 0)
    bound = GROUP_MOVE if igr else PHASE_MOVE
    assert np.all(np.abs(got[moved] / ref[moved] - 1) <= bound)
    return moved.size


@pytest.mark.parametrize("iwave,igr", COMBOS)
def test_plain_form_matches_oracle(oracle, iwave, igr):
    case = S.subgrid(S.config0(), 4, 3)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    pv, svs, svp, srh = dk.depthkernel_vpvsrho(nx, ny, nz, case.vel, case.vp, case.rho, iwave, igr,
                                               K, case.periods, case.depz, case.minthk,
                                               form=dk.FORM_PLAIN)
    ref = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                             rho=case.rho, iwave=iwave, igr=igr)
    assert (ref["status"] == 0).all()
    _moves_ok(pv, ref["pvRc"], iwave, igr)
    tol = GROUP_MOVE / 2 if igr else PHASE_MOVE
    cols = [(svs, ref["sen_vs"], case.vel), (svp, ref["sen_vp"], case.vp),
            (srh, ref["sen_rho"], case.rho)]
    nxy = nx * ny
    for got, exp, x in cols:
        xc = np.asarray(x).reshape(nxy, nz, order="F")
        for c in range(nxy):
            assert_fd_parity(got[c], exp[c], xc[c], tol=tol, max_frac=0.05)


@pytest.mark.parametrize("iwave,igr", COMBOS)
def test_phase_only_table_path_equals_plain_form(oracle, iwave, igr):
    """kernels=False runs the per-column root kernel over the layer tables
    (one thread per column); its velocities equal the plain form's base
    model bit for bit."""
    case = S.subgrid(S.config1(), 8, 6)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    (pv,) = dk.depthkernel(nx, ny, nz, case.vel, iwave, igr, K, case.periods, case.depz,
                           case.minthk, form=dk.FORM_PLAIN, kernels=False)
    pvf, _, _, _ = dk.depthkernel(nx, ny, nz, case.vel, iwave, igr, K, case.periods, case.depz,
                                  case.minthk, form=dk.FORM_PLAIN)
    np.testing.assert_array_equal(pv, pvf)
    ref = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, iwave=iwave,
                             igr=igr, kernels=False)
    _moves_ok(pv, ref["pvRc"], iwave, igr)


def test_gpu_matches_reference_surf96_golden():
    """The Yunnan columns of tests/golden/surf96_wave.npz as a 1-row grid:
    Love / Rayleigh phase and group velocity against the reference's Python
    surf96 (an independent implementation: within the root tolerance)."""
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    g = np.load(os.path.join(here, "golden", "surf96_wave.npz"))
    y = np.load(os.path.join(here, "golden", "yunnan_pv.npz"))
    nx0, ny0, nz = (int(y[k]) for k in ("nx", "ny", "nz"))
    cols = y["vel"].reshape(nx0 * ny0, nz, order="F")[g["columns"]]
    n = cols.shape[0]
    vel = np.asfortranarray(cols.reshape(n, 1, nz))
    t = g["periods"]
    for iwave in (1, 2):
        for igr in (0, 1):
            (pv,) = dk.depthkernel(n, 1, nz, vel, iwave, igr, t.size, t, y["depz"],
                                   float(y["minthk"]), form=dk.FORM_PLAIN, kernels=False)
            ref = g[f"cg_ifunc{iwave}_itype{igr}"]
            rel = np.abs(pv / ref - 1)
            assert rel.max() <= (GROUP_MOVE if igr else PHASE_MOVE), (iwave, igr, rel.max())


def _per_column_oracle(oracle, b, iwave, igr, cols):
    out = []
    for c in cols:
        n0, n1 = b.node_off[c], b.node_off[c + 1]
        p0, p1 = b.per_off[c], b.per_off[c + 1]
        vel = np.asfortranarray(b.vs[n0:n1].reshape(1, 1, n1 - n0))
        out.append(oracle.depthkernel(vel, b.depz[n0:n1], b.periods[p0:p1], b.minthk,
                                      iwave=iwave, igr=igr))
    return out


@pytest.mark.parametrize("iwave,igr", [(2, 1), (1, 0), (1, 1)])
def test_uneven_batch_love_group(oracle, iwave, igr):
    """The uneven-column entry with the form flags: plain-form kernels and
    phase-only runs, per column against the oracle."""
    b = S.config3(realisations=1, columns=48, base_seed=2024)
    flags = (dk.FORM_LOVE if iwave == 1 else 0) | (dk.FORM_GROUP if igr else 0)
    r = depthkernel_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                          form=dk.FORM_PLAIN | flags, kernels=True, lsen=False)
    r0 = depthkernel_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                           form=dk.FORM_PLAIN | flags, kernels=False, lsen=False)
    np.testing.assert_array_equal(r["pv"], r0["pv"])
    assert (r["status"] == 0).all()
    cols = list(range(0, 48, 6))
    refs = _per_column_oracle(oracle, b, iwave, igr, cols)
    tol = GROUP_MOVE / 2 if igr else PHASE_MOVE
    for c, ref in zip(cols, refs):
        pv, svs, svp, srh = r.column(c)
        _moves_ok(pv, ref["pvRc"][0], iwave, igr)
        n0, n1 = b.node_off[c], b.node_off[c + 1]
        vs = b.vs[n0:n1]
        vp, rho = oracle.brocher(vs)
        for got, exp, x in ((svs, ref["sen_vs"][0], vs), (svp, ref["sen_vp"][0], vp),
                            (srh, ref["sen_rho"][0], rho)):
            assert_fd_parity(got, exp, x, tol=tol, max_frac=0.05)


def test_wave_flags_rejected_where_rayleigh_phase_only():
    b = S.config3(realisations=1, columns=4, base_seed=7)
    args = (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    for form, kw in ((dk.FORM_ADJOINT | dk.FORM_LOVE, dict(lsen=True)),   # Lsen: Rayleigh only
                     (dk.FORM_ADJOINT | dk.FORM_GROUP, dict(lsen=True)),
                     (dk.FORM_ADJOINT | dk.FORM_GROUP | dk.FORM_SCAN_FP32, {}),  # FP32 scan: phase
                     (dk.FORM_PLAIN | dk.FORM_LOVE, dict(lsen=True, kernels=False))):
        with pytest.raises(dk.DaziError) as ei:
            depthkernel_batch(*args, form=form, **kw)
        assert ei.value.code == -1


@pytest.mark.parametrize("make", [lambda: S.subgrid(S.config0(), 4, 3),
                                  lambda: S.subgrid(S.config1(), 4, 3)])
def test_love_adjoint_matches_exact_derivative(oracle, make):
    """Adjoint form for Love phase velocity against the oracle's
    high-accuracy central differences (double-precision model pipeline, root
    converged to 1e-13, dln = 1e-4), and against the reference's own kernels
    within their own finite-difference noise.  Love waves do not see Vp: the adjoint's dc/dVp is
    exactly zero (the differences show only round-off)."""
    from conftest import rel_l2
    case = make()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    if case.vp is not None:
        pv, svs, svp, srh = dk.depthkernel_vpvsrho(nx, ny, nz, case.vel, case.vp, case.rho, 1, 0, K,
                                                   case.periods, case.depz, case.minthk,
                                                   form=dk.FORM_ADJOINT)
    else:
        pv, svs, svp, srh = dk.depthkernel(nx, ny, nz, case.vel, 1, 0, K, case.periods,
                                           case.depz, case.minthk, form=dk.FORM_ADJOINT)
    fine = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                              rho=case.rho, iwave=1, tol=1e-13, exact=True, dln=1e-4)
    plain = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                               rho=case.rho, iwave=1)
    assert (plain["status"] == 0).all()
    _moves_ok(pv, plain["pvRc"], 1, 0)
    assert np.count_nonzero(svp) == 0
    assert np.abs(fine["sen_vp"]).max() <= 1e-6 * np.abs(fine["sen_vs"]).max()
    nxy = nx * ny
    worst = {n: max(rel_l2(g[c], fine[k][c]) for c in range(nxy))
             for n, g, k in (("vs", svs, "sen_vs"), ("rho", srh, "sen_rho"))}
    print("Love adjoint vs fine FD worst per-column rel-L2", worst)
    for n, w in worst.items():
        assert w <= 1e-5, (n, w)
    # The reference's kernels difference FP32-rounded phase velocities at
    # dln = 0.01; Love waves are weakly sensitive to density, so that noise
    # is relatively large in dc/drho.  The adjoint must sit as close to the
    # reference's kernels as the exact derivative does.
    for n, g, k in (("vs", svs, "sen_vs"), ("rho", srh, "sen_rho")):
        for c in range(nxy):
            noise = rel_l2(plain[k][c], fine[k][c])
            assert rel_l2(g[c], plain[k][c]) <= 1.5 * noise + 1e-5, (n, c, noise)


def test_love_adjoint_uneven_batch(oracle):
    """The uneven-column entry with FORM_ADJOINT | FORM_LOVE, per column
    against the oracle's high-accuracy differences."""
    from conftest import rel_l2
    b = S.config3(realisations=1, columns=48, base_seed=2024)
    r = depthkernel_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                          form=dk.FORM_ADJOINT | dk.FORM_LOVE, kernels=True, lsen=False)
    assert (r["status"] == 0).all()
    assert np.count_nonzero(r["sen_vp"]) == 0
    for c in range(0, 48, 6):
        n0, n1 = b.node_off[c], b.node_off[c + 1]
        p0, p1 = b.per_off[c], b.per_off[c + 1]
        vel = np.asfortranarray(b.vs[n0:n1].reshape(1, 1, n1 - n0))
        fine = oracle.depthkernel(vel, b.depz[n0:n1], b.periods[p0:p1], b.minthk, iwave=1,
                                  tol=1e-13, exact=True, dln=1e-4)
        pv, svs, svp, srh = r.column(c)
        assert rel_l2(svs, fine["sen_vs"][0]) <= 1e-5, c
        assert rel_l2(srh, fine["sen_rho"][0]) <= 1e-5, c


def _group_fd_pair(oracle, vel, depz, periods, minthk, iwave, vp=None, rho=None):
    """The oracle's exact-model group velocity differenced at dln = 1e-4 and
    4e-4.  The quotient over t/(1 -+ h) amplifies root round-off ~1/(2h) =
    100-fold, so the two differ by the differences' own noise (largest in
    the weakly sensitive density kernels)."""
    kw = dict(vp=vp, rho=rho, iwave=iwave, igr=1, tol=1e-13, exact=True)
    return (oracle.depthkernel(vel, depz, periods, minthk, dln=1e-4, **kw),
            oracle.depthkernel(vel, depz, periods, minthk, dln=4e-4, **kw))


def _assert_group_kernels(rel_l2, got, f1, f2, c, names):
    """Per column: within 3x the exact differences' own noise (+1e-6), and
    within the 1e-4 rel-L2 kernel bar."""
    for n in names:
        noise = rel_l2(f1["sen_" + n][c], f2["sen_" + n][c])
        err = rel_l2(got[n], f1["sen_" + n][c])
        assert err <= min(3.0 * noise + 1.0e-6, 1.0e-4), (n, c, err, noise)


@pytest.mark.parametrize("iwave", [2, 1])
@pytest.mark.parametrize("make", [lambda: S.subgrid(S.config0(), 4, 3),
                                  lambda: S.subgrid(S.config1(), 4, 3)])
def test_group_adjoint_matches_exact_derivative(oracle, make, iwave):
    """Adjoint form for group velocity: the derivative of the reference's
    quotient of the roots at t1a and t1b, from phase adjoints at both,
    against the oracle's exact-model differences of the same quotient."""
    from conftest import rel_l2
    case = make()
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    if case.vp is not None:
        pv, svs, svp, srh = dk.depthkernel_vpvsrho(nx, ny, nz, case.vel, case.vp, case.rho, iwave,
                                                   1, K, case.periods, case.depz, case.minthk,
                                                   form=dk.FORM_ADJOINT)
    else:
        pv, svs, svp, srh = dk.depthkernel(nx, ny, nz, case.vel, iwave, 1, K, case.periods,
                                           case.depz, case.minthk, form=dk.FORM_ADJOINT)
    plain = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                               rho=case.rho, iwave=iwave, igr=1)
    assert (plain["status"] == 0).all()
    _moves_ok(pv, plain["pvRc"], iwave, 1)
    f1, f2 = _group_fd_pair(oracle, case.vel, case.depz, case.periods, case.minthk, iwave,
                            vp=case.vp, rho=case.rho)
    names = ("vs", "rho") if iwave == 1 else ("vs", "vp", "rho")
    if iwave == 1:
        assert np.count_nonzero(svp) == 0
    for c in range(nx * ny):
        got = {"vs": svs[c], "vp": svp[c], "rho": srh[c]}
        _assert_group_kernels(rel_l2, got, f1, f2, c, names)


@pytest.mark.parametrize("iwave", [2, 1])
def test_group_adjoint_uneven_batch(oracle, iwave):
    """The uneven-column entry with FORM_ADJOINT | FORM_GROUP (| FORM_LOVE),
    per column against the oracle's exact-model differences."""
    from conftest import rel_l2
    b = S.config3(realisations=1, columns=48, base_seed=2024)
    form = dk.FORM_ADJOINT | dk.FORM_GROUP | (dk.FORM_LOVE if iwave == 1 else 0)
    r = depthkernel_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                          form=form, kernels=True, lsen=False)
    assert (r["status"] == 0).all()
    names = ("vs", "rho") if iwave == 1 else ("vs", "vp", "rho")
    for c in range(0, 48, 6):
        n0, n1 = b.node_off[c], b.node_off[c + 1]
        p0, p1 = b.per_off[c], b.per_off[c + 1]
        vel = np.asfortranarray(b.vs[n0:n1].reshape(1, 1, n1 - n0))
        f1, f2 = _group_fd_pair(oracle, vel, b.depz[n0:n1], b.periods[p0:p1], b.minthk, iwave)
        pv, svs, svp, srh = r.column(c)
        _assert_group_kernels(rel_l2, {"vs": svs, "vp": svp, "rho": srh}, f1, f2, 0, names)
