"""tregn96's partials checked against a second code path (CPU, oracle only).

The Gc/Gs kernel Lsen_Gsc is built from tregn96's energy-integral partials
dcdah, dcdav, dcdbh, dcdbv, dcdn (svfunc -> down -> energy/intijr ->
getdcdh, tregn96.f:1559-1832, 3561-3709, 3777-4377), then gammap's Q shift
of c (:3711-3775), sprayl's sphericity scaling (:1235-1299) and
depthkernelTI's splice (depthkernelTI.f90:124-162).  No reference fixture
holds any of these, so each link is checked here against something that
does not go through the energy integrals:

1. The TI secular function (the top entry of up()'s compound vector,
   tregn96.f:1834-1990, through gettiegn/varsv/dnka_tregn) has, at
   isotropic moduli, the same root as surfdisp96's dltar4 (whose phase
   velocities reproduce the reference's golden output file).
2. Central differences of that TI root with respect to A, C, F, L, N of one
   layer (rho fixed) equal the partials converted to moduli:
       dc/dA = dcdah/(2 rho alpha_h) - F/(A - 2L)^2 dcdn
       dc/dC = dcdav/(2 rho alpha_v)
       dc/dF = dcdn/(A - 2L)
       dc/dL = dcdbv/(2 rho beta_v) + 2F/(A - 2L)^2 dcdn
       dc/dN = dcdbh/(2 rho beta_h)   (zero: Rayleigh waves do not see N)
   (A = rho alpha_h^2, C = rho alpha_v^2, L = rho beta_v^2,
   N = rho beta_h^2, F = eta (A - 2L)), on the flat config-0 model, on a
   transversely isotropic variant of it and on 20 seeded config-3 columns.
3. sprayl: with sphericity the alpha/beta partials are the flat model's
   times vtp/tm^3 and dcdn is left unscaled.
4. gammap: the Q shift adds sum (dcdb* beta qbi + dcda* alpha qai)
   ln(omega/omega_ref)/pi to c and leaves the partials unchanged.
5. The splice: sum over an interval's sublayers of A dc/dA + L dc/dL equals
   the difference of the TI root when A and L of those sublayers are scaled
   together; and the oracle's Lsen_Gsc is that sum of its real*4 partials
   in real*4, in the order of depthkernelTI.f90:152-162.
"""
import numpy as np

from dazi_current_release_b200 import synthetic as S

TWOPI32 = np.float32(2.0) * np.float32(3.141592654)     # tregn96's real*4 twopi
H = 1e-5                                                  # relative step of the differences
PARTIAL_TOL = 1e-6                                        # rel-L2 per (column, period, modulus)


def _ti_model(O, depz, vs, minthk, ani=None):
    """depthkernelTI's layer moduli (depthkernelTI.f90:124-131), real*4.
    ani = (c_over_a, n_over_l, eta) makes a transversely isotropic variant."""
    vp, rho = O.brocher(np.asarray(vs, np.float32))
    thk, rvp, rvs, rrho, nsub = O.refine(minthk, depz, vp, vs, rho)
    TA = (rrho * (rvp * rvp)).astype(np.float32)
    TL = (rrho * (rvs * rvs)).astype(np.float32)
    TF = (np.float32(1.0) * (TA - np.float32(2.0) * TL)).astype(np.float32)
    TC, TN = TA.copy(), TL.copy()
    if ani is not None:
        TC = (TA * np.float32(ani[0])).astype(np.float32)
        TN = (TL * np.float32(ani[1])).astype(np.float32)
        TF = (np.float32(ani[2]) * (TA - np.float32(2.0) * TL)).astype(np.float32)
    return dict(thk=thk, TA=TA, TC=TC, TF=TF, TL=TL, TN=TN, rho=rrho, nsub=nsub, vp=rvp, vs=rvs)


def _moduli(m):
    return [m[k] for k in ("thk", "TA", "TC", "TF", "TL", "TN", "rho")]


def _omega(t):
    return float(TWOPI32) / float(np.float32(t))


def _converted(full, m):
    """tregn96's FP64 partials (ah, av, bh, bv, n) as dc/d(A, C, F, L, N)."""
    ah, av, bh, bv, n = full[:5]
    A, C, F, L, N, R = (m[k].astype(np.float64) for k in ("TA", "TC", "TF", "TL", "TN", "rho"))
    g = A - 2 * L
    return np.stack([ah / (2 * R * np.sqrt(A / R)) - F / g ** 2 * n,
                     av / (2 * R * np.sqrt(C / R)),
                     n / g,
                     bv / (2 * R * np.sqrt(L / R)) + 2 * F / g ** 2 * n,
                     bh / (2 * R * np.sqrt(N / R))])


def _root(O, m, t, guess):
    return O.ti_root(*_moduli(m), _omega(t), guess, xtol=1e-15)


def _check_partials(O, m, periods, layers, guesses):
    """Returns the worst rel-L2 over the periods and the moduli A, C, F, L,
    and the largest |dc/dN| relative to max |dc/dA|."""
    worst, worst_n = 0.0, 0.0
    for t, g in zip(periods, guesses):
        c = _root(O, m, t, g)
        full = O.tregn96(*_moduli(m), [np.float32(t)], [c], nsph=0, dogam=0, full=True,
                         cp_double=True)[3][0]
        an = _converted(full, m)[:, layers]
        perts = [(l, l, k) for k in range(5) for l in layers]
        fd = O.ti_root_fd(*_moduli(m), _omega(t), c, perts, h=H).reshape(5, len(layers))
        for k in range(4):
            worst = max(worst, np.linalg.norm(fd[k] - an[k]) / np.linalg.norm(fd[k]))
        scale = np.abs(an[0]).max()
        worst_n = max(worst_n, np.abs(fd[4]).max() / scale, np.abs(an[4]).max() / scale)
    return worst, worst_n


def _config0_column():
    c0 = S.config0()
    return c0.depz, c0.vel[0, 0, :], c0.minthk, c0.periods


def _config3_columns(n=20, seed=99):
    b = S.config3(realisations=1, columns=2500)
    idx = np.sort(np.random.default_rng(seed).choice(b.ncol, n, replace=False))
    return [b.column(int(c)) for c in idx], b.minthk


def _flat_guess(O, m, periods):
    """surfdisp96's exact flat-earth root at tregn96's omega, as the start."""
    return O.surfdisp96_d(m["thk"], m["vp"], m["vs"], m["rho"],
                          [2 * np.pi / _omega(t) for t in periods], iflsph=0, tol=1e-14)[0]


def test_ti_secular_root_equals_isotropic_root(oracle):
    """Link 1: at isotropic moduli formed in double, the TI root is
    surfdisp96's root (both flat, both to 1e-15)."""
    O = oracle
    cols = [_config0_column()[:3] + (S.config0().periods,)]
    c3, mt = _config3_columns(5, seed=5)
    cols += [(d, v, mt, p) for d, v, p in c3]
    worst = 0.0
    for depz, vs, minthk, periods in cols:
        vp, rho = O.brocher(np.asarray(vs, np.float32))
        thk, rvp, rvs, rrho, _ = O.refine(minthk, depz, vp, vs, rho)
        R, a, b = (x.astype(np.float64) for x in (rrho, rvp, rvs))
        A, L = R * a * a, R * b * b
        cg, st = O.surfdisp96_d(thk, rvp, rvs, rrho, periods, iflsph=0, tol=1e-15)
        for t, c in zip(periods, cg):
            if c <= 0:
                continue
            cr = O.ti_root(thk, A, A, A - 2 * L, L, L, R, 2 * np.pi / t, c, xtol=1e-15)
            worst = max(worst, abs(cr / c - 1))
    assert worst <= 1e-12, worst


def test_partials_match_root_differences_flat_model(oracle):
    """Link 2 on the flat config-0 model: every period, every 4th layer and
    the half-space."""
    O = oracle
    depz, vs, minthk, periods = _config0_column()
    m = _ti_model(O, depz, vs, minthk)
    nl = m["thk"].size
    layers = list(range(0, nl - 1, 4)) + [nl - 1]
    worst, worst_n = _check_partials(O, m, periods, layers, _flat_guess(O, m, periods))
    assert worst <= PARTIAL_TOL, worst
    assert worst_n <= 1e-12, worst_n


def test_partials_match_root_differences_ti_model(oracle):
    """Link 2 on a transversely isotropic variant (C = 0.95 A, N = 1.08 L,
    eta = 0.9): the TI-specific terms of the eigen-solution and integrals."""
    O = oracle
    depz, vs, minthk, periods = _config0_column()
    m = _ti_model(O, depz, vs, minthk, ani=(0.95, 1.08, 0.9))
    nl = m["thk"].size
    layers = list(range(0, nl - 1, 5)) + [nl - 1]
    sel = periods[::3]
    worst, worst_n = _check_partials(O, m, sel, layers, _flat_guess(O, m, sel))
    assert worst <= PARTIAL_TOL, worst
    assert worst_n <= 1e-12, worst_n


def test_partials_match_root_differences_config3(oracle):
    """Link 2 on 20 seeded columns of the uneven workload (sediments, some
    low-velocity zones): 4 periods each, up to 24 layers spread over the
    stack including the half-space."""
    O = oracle
    cols, minthk = _config3_columns(20)
    worst_all, worst_n_all = 0.0, 0.0
    for depz, vs, periods in cols:
        m = _ti_model(O, depz, vs, minthk)
        nl = m["thk"].size
        layers = sorted(set(np.linspace(0, nl - 1, min(24, nl)).astype(int).tolist()))
        sel = periods[np.linspace(0, periods.size - 1, 4).astype(int)]
        guess = _flat_guess(O, m, sel)
        if (guess <= 0).any():
            continue
        w, wn = _check_partials(O, m, sel, layers, guess)
        worst_all, worst_n_all = max(worst_all, w), max(worst_n_all, wn)
    assert worst_all <= PARTIAL_TOL, worst_all
    assert worst_n_all <= 1e-12, worst_n_all


def _flatten(m):
    """sphere_tdisp96 (tregn96.f:774-841), Rayleigh: thicknesses to
    ar ln(ar/r), rho x tmp^-2.275, moduli x tmp^-0.275, real*4 stores; and
    bldsph's (:1301-1383) vtp from the flattened thicknesses."""
    ar = 6371.0
    d = m["thk"].astype(np.float32).copy()
    d[-1] = np.float32(1.0)
    out = {k: m[k].copy() for k in ("TA", "TC", "TF", "TL", "TN", "rho")}
    r0 = ar
    fl = np.zeros_like(d)
    for i in range(d.size):
        r1 = r0 - float(d[i])
        z0, z1 = ar * np.log(ar / r0), ar * np.log(ar / r1)
        fl[i] = np.float32(z1 - z0)
        tmp = (ar + ar) / (r0 + r1)
        out["rho"][i] = np.float32(float(m["rho"][i]) * tmp ** float(np.float32(-2.275)))
        f275 = tmp ** float(np.float32(-0.275))
        for k in ("TA", "TC", "TL", "TN"):
            out[k][i] = np.float32(float(m[k][i]) * f275)
        r0 = r1
    fl[-1] = np.float32(0.0)
    out["thk"] = fl
    ars = 6370.0
    zd = fl.astype(np.float64)
    zd[-1] = 1.0
    vtp = np.zeros(d.size, np.float32)
    r0 = ars
    for i in range(d.size):
        r1 = r0 * np.exp(-zd[i] / ars)
        vtp[i] = np.float32((ars + ars) / (r0 + r1))
        r0 = r1
    return out, vtp


def test_sprayl_scales_alpha_beta_partials_not_eta(oracle):
    """Link 3: tregn96 with sphericity = the flattened model's partials
    (no sphericity) x vtp/tm^3 for ah, av, bh, bv; dcdn unscaled."""
    O = oracle
    depz, vs, minthk, periods = _config0_column()
    m = _ti_model(O, depz, vs, minthk)
    flat, vtp = _flatten(m)
    cp = _flat_guess(O, m, periods)
    t32 = periods.astype(np.float32)
    sph = O.tregn96(*_moduli(m), t32, cp, nsph=1, dogam=0, full=True, cp_double=True)[3]
    fla = O.tregn96(*[flat[k] for k in ("thk", "TA", "TC", "TF", "TL", "TN", "rho")], t32, cp,
                    nsph=0, dogam=0, full=True, cp_double=True)[3]
    for k, t in enumerate(t32):
        om = _omega(t)
        tm = np.sqrt(1.0 + (cp[k] / (2.0 * 6370.0 * om)) ** 2)
        for j in range(4):          # ah, av, bh, bv
            exp = fla[k, j] * vtp.astype(np.float64) / tm ** 3
            den = np.abs(exp).max()
            if den > 0:
                assert np.abs(sph[k, j] - exp).max() <= 1e-6 * den, (k, j)
        np.testing.assert_allclose(sph[k, 4], fla[k, 4], rtol=1e-6,
                                   atol=1e-6 * np.abs(fla[k, 4]).max())


def test_gammap_shifts_c_and_keeps_partials(oracle):
    """Link 4: Q = 150/50, reference frequency 1 Hz (depthkernelTI.f90:
    132-137); gammap's pi is the reference's 3.141592653589493."""
    O = oracle
    depz, vs, minthk, periods = _config0_column()
    m = _ti_model(O, depz, vs, minthk)
    cp = _flat_guess(O, m, periods)
    t32 = periods.astype(np.float32)
    q = O.tregn96(*_moduli(m), t32, cp, nsph=0, dogam=1, full=True, cp_double=True)[3]
    e = O.tregn96(*_moduli(m), t32, cp, nsph=0, dogam=0, full=True, cp_double=True)[3]
    np.testing.assert_array_equal(q[:, :6], e[:, :6])
    R = m["rho"].astype(np.float64)
    ah, av = np.sqrt(m["TA"] / R), np.sqrt(m["TC"] / R)
    bh, bv = np.sqrt(m["TN"] / R), np.sqrt(m["TL"] / R)
    pi_ref = 3.141592653589493
    qai = float(np.float32(1.0) / np.float32(150.0))    # 1/Q stored as real*4
    qbi = float(np.float32(1.0) / np.float32(50.0))
    for k, t in enumerate(t32):
        lw = np.log(_omega(t) / (2.0 * pi_ref * 1.0)) / pi_ref
        dc = (lw * ((e[k, 2] * bh + e[k, 3] * bv) * qbi)).sum() + \
             (lw * ((e[k, 1] * av + e[k, 0] * ah) * qai)).sum()
        assert abs(q[k, 6, 0] - (cp[k] + dc)) <= 1e-12 * cp[k]
        assert q[k, 6, 0] < cp[k]        # periods longer than 1 s: below the 1 Hz velocity


def test_splice_sum_matches_root_difference(oracle):
    """Link 5a: per depth interval, sum over its sublayers of A dc/dA +
    L dc/dL (the splice's combination, depthkernelTI.f90:152-158) equals the
    central difference of the TI root with A and L of those sublayers scaled
    by (1 +- h)."""
    O = oracle
    depz, vs, minthk, periods = _config0_column()
    m = _ti_model(O, depz, vs, minthk)
    starts = np.concatenate([[0], np.cumsum(m["nsub"])])
    A, L = m["TA"].astype(np.float64), m["TL"].astype(np.float64)
    cp = _flat_guess(O, m, periods)
    worst = 0.0
    for k in (0, 4, 9):
        c = _root(O, m, periods[k], cp[k])
        full = O.tregn96(*_moduli(m), [np.float32(periods[k])], [c], nsph=0, dogam=0,
                         full=True, cp_double=True)[3][0]
        d = _converted(full, m)
        per_layer = A * d[0] + L * d[3]
        exp = np.array([per_layer[starts[j]:starts[j + 1]].sum() for j in range(len(m["nsub"]))])
        perts = [(int(starts[j]), int(starts[j + 1]) - 1, 5) for j in range(len(m["nsub"]))]
        fd = O.ti_root_fd(*_moduli(m), _omega(periods[k]), c, perts, h=H)
        worst = max(worst, np.linalg.norm(fd - exp) / np.linalg.norm(fd))
    assert worst <= PARTIAL_TOL, worst


def test_oracle_lsen_is_the_real4_splice_of_its_partials(oracle):
    """Link 5b: or_depthkernelTI's Lsen_Gsc equals depthkernelTI.f90:152-162
    applied in real*4 to or_tregn96's real*4 partials at the real*4 phase
    velocities (sphericity and Q on, as the reference calls it)."""
    O = oracle
    c0 = S.subgrid(S.config0(), 2, 1)
    ref = O.depthkernel_ti(c0.vel, c0.depz, c0.periods, c0.minthk)
    f32 = np.float32
    for col in range(2):
        m = _ti_model(O, c0.depz, c0.vel.reshape(2, -1, order="F")[col], c0.minthk)
        cp = ref["pvRc"][col].astype(np.float32)
        dah, dbv, dn = O.tregn96(*_moduli(m), c0.periods.astype(np.float32), cp)
        TA, TL, TF, R = m["TA"], m["TL"], m["TF"], m["rho"]
        rvp, rvs = m["vp"], m["vs"]
        for i in range(c0.periods.size):
            k = 0
            for j, ns in enumerate(m["nsub"]):
                acc = f32(0.0)
                for _ in range(ns):
                    tfd = f32(TA[k] - f32(2.0) * TL[k])
                    dA = f32(f32(f32(0.5) / f32(R[k] * rvp[k])) * dah[i, k]) - \
                        f32(f32(TF[k] / f32(tfd * tfd)) * dn[i, k])
                    dL = f32(f32(f32(0.5) / f32(R[k] * rvs[k])) * dbv[i, k]) + \
                        f32(f32(f32(f32(2.0) * TF[k]) / f32(tfd * tfd)) * dn[i, k])
                    acc = f32(f32(acc + f32(dA * TA[k])) + f32(dL * TL[k]))
                    k += 1
                assert ref["Lsen_Gsc"][col, i, j] == acc, (col, i, j)
