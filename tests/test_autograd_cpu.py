"""Host-side bookkeeping of the torch binding (no device needed): the maps
from kernel entries to (period, node) and from Lsen entries to (period,
interval), the vector-Jacobian product and the azimuthal epilogue, against
explicit loops over the batch layout."""
import numpy as np
import torch

from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.autograd import (ColumnBatch, azimuthal_phase_velocity,
                                                brocher_derivatives)


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
