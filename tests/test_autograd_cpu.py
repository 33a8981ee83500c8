"""Host-side bookkeeping of the torch binding (no device needed): the maps
from kernel entries to (period, node) and from Lsen entries to (period,
interval), the vector-Jacobian product and the azimuthal epilogue, against
explicit loops over the batch layout; the autograd functions with the
library call replaced by fixed kernels."""
import numpy as np
import torch

from dazi_current_release_b200 import synthetic as S
import pytest

from dazi_current_release_b200 import _lib
from dazi_current_release_b200.autograd import (ColumnBatch, azimuthal_phase_velocity,
                                                brocher_derivatives, dispersion_velocity,
                                                phase_velocity)


def _batch():
    b = S.config3(realisations=1, columns=7, base_seed=1000)
    return b, ColumnBatch(b.node_off, b.depz, b.per_off, b.periods, b.minthk, device="cpu")


def test_vjp_matches_loops():
    b, cb = _batch()
    rng = np.random.default_rng(0)
    g = rng.standard_normal(cb.nper)
    kern = rng.standard_normal(cb.nsen)
    got = cb.vjp(torch.as_tensor(g), torch.as_tensor(kern)).numpy()
    exp = np.zeros(cb.nnodes)
    so = 0
    for c in range(b.ncol):
        K = b.per_off[c + 1] - b.per_off[c]
        nz = b.node_off[c + 1] - b.node_off[c]
        for i in range(nz):
            for k in range(K):
                exp[b.node_off[c] + i] += g[b.per_off[c] + k] * kern[so + k + K * i]
        so += K * nz
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)


def test_azimuthal_epilogue_matches_loops():
    b, cb = _batch()
    rng = np.random.default_rng(1)
    c0 = torch.as_tensor(rng.uniform(2, 4, cb.nper))
    ls = torch.as_tensor(rng.standard_normal(cb.nls).astype(np.float32))
    gc = torch.as_tensor(rng.standard_normal(cb.nintervals))
    gs = torch.as_tensor(rng.standard_normal(cb.nintervals))
    psi = torch.as_tensor(rng.uniform(0, np.pi, cb.nper))
    got = azimuthal_phase_velocity(c0, ls, gc, gs, psi, cb).numpy()
    exp = c0.numpy().copy()
    lo = 0
    for c in range(b.ncol):
        K = b.per_off[c + 1] - b.per_off[c]
        nz = b.node_off[c + 1] - b.node_off[c]
        j0 = b.node_off[c] - c
        for j in range(nz - 1):
            for k in range(K):
                p = b.per_off[c] + k
                exp[p] += float(ls[lo + k + K * j]) * (gc[j0 + j].item() * np.cos(2 * psi[p].item())
                                                      + gs[j0 + j].item() * np.sin(2 * psi[p].item()))
        lo += K * (nz - 1)
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)


def test_brocher_derivatives_match_fd():
    vs = torch.linspace(0.8, 4.8, 41, dtype=torch.float64)
    dvp, drho = brocher_derivatives(vs)

    def f(v):
        vp = 0.9409 + 2.0947 * v - 0.8206 * v ** 2 + 0.2683 * v ** 3 - 0.0251 * v ** 4
        rho = 1.6612 * vp - 0.4721 * vp ** 2 + 0.0671 * vp ** 3 - 0.0043 * vp ** 4 + 0.000106 * vp ** 5
        return vp, rho

    h = 1e-6
    (p1, r1), (p0, r0) = f(vs + h), f(vs - h)
    torch.testing.assert_close(dvp, (p1 - p0) / (2 * h), rtol=1e-7, atol=1e-8)
    torch.testing.assert_close(drho, (r1 - r0) / (2 * h), rtol=1e-7, atol=1e-8)


def _stub_run(cb, calls):
    """Replaces the library call of cb by fixed kernels, recording flags."""
    rng = np.random.default_rng(2)
    sen = [torch.as_tensor(rng.standard_normal(cb.nsen)) for _ in range(3)]
    pv = torch.as_tensor(rng.uniform(2.0, 4.0, cb.nper))

    def run(vs, vp=None, rho=None, lsen=True, flags=0):
        calls.append((lsen, flags))
        ls = torch.zeros(cb.nls, dtype=torch.float32) if lsen else None
        return pv.clone(), [t.clone() for t in sen], ls, torch.zeros(cb.ncols, dtype=torch.int32)

    cb.run = run
    return pv, sen


@pytest.mark.parametrize("iwave,igr,flags", [(2, 0, 0), (1, 0, _lib.FORM_LOVE),
                                             (2, 1, _lib.FORM_GROUP),
                                             (1, 3, _lib.FORM_LOVE | _lib.FORM_GROUP)])
def test_dispersion_velocity_flags_and_gradient(iwave, igr, flags):
    """iwave/igr become the library's form flags (no Lsen_Gsc with them),
    and the gradient is the VJP of the returned kernels: the total Vs
    derivative through the Brocher relations, or one partial per input."""
    b, cb = _batch()
    calls = []
    pv, sen = _stub_run(cb, calls)
    rng = np.random.default_rng(3)
    w = torch.as_tensor(rng.standard_normal(cb.nper))
    vs = torch.as_tensor(np.asarray(b.vs, np.float32)).requires_grad_(True)
    c, status = dispersion_velocity(vs, cb, iwave=iwave, igr=igr)
    assert calls == [(flags == 0, flags)]
    torch.testing.assert_close(c, pv)
    (c * w).sum().backward()
    dvp, drho = brocher_derivatives(vs.detach())
    k_tot = sen[0] + dvp[cb._sen_node] * sen[1] + drho[cb._sen_node] * sen[2]
    torch.testing.assert_close(vs.grad.double(), cb.vjp(w, k_tot).to(torch.float32).double())
    # explicit Vp and rho: one partial kernel each
    vp = (1.75 * vs.detach()).requires_grad_(True)
    rho = torch.full_like(vp, 2.7).requires_grad_(True)
    vs.grad = None
    c, _ = dispersion_velocity(vs, cb, vp=vp, rho=rho, iwave=iwave, igr=igr)
    (c * w).sum().backward()
    for x, k in ((vs, sen[0]), (vp, sen[1]), (rho, sen[2])):
        torch.testing.assert_close(x.grad, cb.vjp(w, k).to(torch.float32))


def test_phase_velocity_keeps_lsen_and_rejects_bad_arguments():
    b, cb = _batch()
    calls = []
    _stub_run(cb, calls)
    vs = torch.as_tensor(np.asarray(b.vs, np.float32))
    c0, ls, status = phase_velocity(vs, cb)
    assert calls == [(True, 0)] and ls.numel() == cb.nls
    with pytest.raises(ValueError):
        dispersion_velocity(vs, cb, iwave=3)
    with pytest.raises(ValueError):
        dispersion_velocity(vs, cb, vp=vs)
