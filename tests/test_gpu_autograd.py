"""Differentiation (config 2 recipe): loss = sum of squared misfits between
the predicted c(T) (with the azimuthal term of Gc/Gs) and "observed" phase
velocities of a 3 %-perturbed model, differentiated by the torch binding
whose backward is the library's adjoint form.

d loss / dVs is checked against central finite differences in FP64 with
relative step 1e-4 (the oracle's exact double pipeline, root converged to
1e-13, chained through the Brocher relations) and against the reference's
own perturb-and-recompute kernels (within the reference's A/B gate); d loss
/ dGc, dGs against the oracle's Lsen_Gsc."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from dazi_current_release_b200 import synthetic as S
from dazi_current_release_b200.autograd import (ColumnBatch, azimuthal_phase_velocity,
                                                brocher_derivatives, dispersion_velocity,
                                                phase_velocity)

pytestmark = pytest.mark.gpu


def _case():
    full = S.config2()
    case = S.subgrid(full, 3, 2)
    obs = np.asfortranarray(full.extra["vs_obs"][:3, :2, :])
    return case, obs


def _flat(vel):
    nx, ny, nz = vel.shape
    return np.ascontiguousarray(vel.reshape(nx * ny, nz, order="F")).ravel()


def test_loss_gradient_matches_fd_and_reference_kernels(oracle):
    case, vs_obs = _case()
    nx, ny, nz = case.vel.shape
    n, K = nx * ny, case.periods.size
    dev = torch.device("cuda")
    batch = ColumnBatch.from_grid(nx, ny, case.depz, case.periods, case.minthk, device=dev)
    c_obs, _, _, st = batch.run(torch.as_tensor(_flat(vs_obs), device=dev))
    assert int(st.abs().sum()) == 0
    vs = torch.tensor(_flat(case.vel), device=dev, requires_grad=True)
    gc = torch.zeros(batch.nintervals, dtype=torch.float64, device=dev, requires_grad=True)
    gs = torch.zeros_like(gc, requires_grad=True)
    psi = torch.as_tensor(np.random.default_rng(4).uniform(0.0, np.pi, batch.nper), device=dev)
    c0, lsen, status = phase_velocity(vs, batch)
    c = azimuthal_phase_velocity(c0, lsen, gc, gs, psi, batch)
    loss = ((c - c_obs) ** 2).sum()
    loss.backward()
    g_vs = vs.grad.double().cpu().numpy().reshape(n, nz)
    resid = (2.0 * (c - c_obs)).detach().cpu().numpy().reshape(n, K)

    # FP64 central differences, relative step 1e-4, chained through Brocher
    fine = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, tol=1e-13,
                              exact=True, dln=1e-4)
    ref = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk)
    dvp, drho = (t.cpu().numpy().reshape(n, nz) for t in
                 brocher_derivatives(torch.as_tensor(_flat(case.vel))))

    def expected(r):
        k = r["sen_vs"] + dvp[:, None, :] * r["sen_vp"] + drho[:, None, :] * r["sen_rho"]
        return np.einsum("ck,ckn->cn", resid, k)

    g_fd, g_ref = expected(fine), expected(ref)
    e_fd = rel_l2(g_vs, g_fd)
    e_ref = rel_l2(g_vs, g_ref)
    print("d loss/dVs: rel-L2 vs FP64 central FD", e_fd, "vs reference kernels", e_ref)
    assert e_fd <= 1e-5
    assert e_ref <= 1e-3

    # Gc/Gs: d loss/dGc_j = sum_k resid_k Lsen_kj cos 2 psi_k (Gc = Gs = 0)
    ti = oracle.depthkernel_ti(case.vel, case.depz, case.periods, case.minthk)
    L = ti["Lsen_Gsc"]                                         # (n, K, nz-1)
    ps = psi.cpu().numpy().reshape(n, K)
    egc = np.einsum("ck,ckj->cj", resid * np.cos(2 * ps), L).ravel()
    egs = np.einsum("ck,ckj->cj", resid * np.sin(2 * ps), L).ravel()
    e_gc = rel_l2(gc.grad.cpu().numpy(), egc)
    e_gs = rel_l2(gs.grad.cpu().numpy(), egs)
    print("d loss/dGc rel-L2", e_gc, "dGs", e_gs)
    assert e_gc <= 1e-5 and e_gs <= 1e-5


def test_explicit_vp_rho_gradients(oracle):
    """With Vp and rho as inputs, each gets its own partial kernel."""
    case = S.subgrid(S.config0(), 3, 2)
    nx, ny, nz = case.vel.shape
    n, K = nx * ny, case.periods.size
    dev = torch.device("cuda")
    batch = ColumnBatch.from_grid(nx, ny, case.depz, case.periods, case.minthk, device=dev)
    t = lambda a: torch.tensor(_flat(a), device=dev, requires_grad=True)  # noqa: E731
    vs, vp, rho = t(case.vel), t(case.vp), t(case.rho)
    w = torch.as_tensor(np.random.default_rng(1).standard_normal(batch.nper), device=dev)
    c0, _, _ = phase_velocity(vs, batch, vp=vp, rho=rho)
    (c0 * w).sum().backward()
    fine = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, vp=case.vp,
                              rho=case.rho, tol=1e-13, exact=True, dln=1e-4)
    wn = w.cpu().numpy().reshape(n, K)
    for x, name in ((vs, "sen_vs"), (vp, "sen_vp"), (rho, "sen_rho")):
        exp = np.einsum("ck,ckn->cn", wn, fine[name])
        e = rel_l2(x.grad.double().cpu().numpy().reshape(n, nz), exp)
        print(name, "VJP rel-L2 vs FP64 central FD", e)
        assert e <= 1e-5


@pytest.mark.parametrize("iwave,igr", [(2, 0), (1, 0), (2, 1), (1, 1)])
def test_dispersion_velocity_gradient(oracle, iwave, igr):
    """Love / Rayleigh, phase / group velocity through the torch binding:
    the gradient of a weighted sum of c against the oracle's exact-model
    differences (root to 1e-13, dln = 1e-4) chained through the Brocher
    relations.  Group velocity's differences carry ~1/(2h) = 100 times the
    root round-off, hence the wider bound (the 1e-4 kernel bar)."""
    case = S.subgrid(S.config1(), 3, 2)
    nx, ny, nz = case.vel.shape
    n, K = nx * ny, case.periods.size
    dev = torch.device("cuda")
    batch = ColumnBatch.from_grid(nx, ny, case.depz, case.periods, case.minthk, device=dev)
    vs = torch.tensor(_flat(case.vel), device=dev, requires_grad=True)
    w = torch.as_tensor(np.random.default_rng(5).standard_normal(batch.nper), device=dev)
    c, status = dispersion_velocity(vs, batch, iwave=iwave, igr=igr)
    assert int(status.abs().sum()) == 0
    (c * w).sum().backward()
    g = vs.grad.double().cpu().numpy().reshape(n, nz)
    plain = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, iwave=iwave, igr=igr)
    move = np.abs(c.detach().cpu().numpy().reshape(n, K) / plain["pvRc"] - 1)
    assert move.max() <= (4.0e-4 if igr else 2.0e-6), move.max()
    fine = oracle.depthkernel(case.vel, case.depz, case.periods, case.minthk, iwave=iwave,
                              igr=igr, tol=1e-13, exact=True, dln=1e-4)
    dvp, drho = (t.cpu().numpy().reshape(n, nz) for t in
                 brocher_derivatives(torch.as_tensor(_flat(case.vel))))
    k_tot = fine["sen_vs"] + dvp[:, None, :] * fine["sen_vp"] + drho[:, None, :] * fine["sen_rho"]
    expect = np.einsum("ck,cki->ci", w.cpu().numpy().reshape(n, K), k_tot)
    worst = max(rel_l2(g[i], expect[i]) for i in range(n))
    print("dispersion_velocity gradient vs exact differences, worst column", iwave, igr, worst)
    assert worst <= (1.0e-4 if igr else 1.0e-5), worst
