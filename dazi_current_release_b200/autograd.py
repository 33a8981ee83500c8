"""PyTorch binding with gradients: phase velocities of a column batch as a
differentiable function of the node velocities (Rayleigh phase velocity
with the Gc/Gs kernel; Love waves and group velocity through
`dispersion_velocity`).

Forward: the library's adjoint form (dazi_dk_batch_dev, form ADJOINT) on the
tensors' CUDA stream computes c(T) for every (column, period), the three
node kernels dc/dVs, dc/dVp, dc/drho (implicit differentiation of the
Rayleigh root, dc/dm = -(dF/dm)/(dF/dc)) and the Gc/Gs kernel Lsen_Gsc.
Backward: the vector-Jacobian product of those kernels with the incoming
gradient of c.  When Vp and rho follow Vs through the Brocher relations
(depthkernel_empirical_vp_rho, DepthKernel1D.f90:187-200), the gradient with
respect to Vs is the total derivative
    dc/dVs + dVp/dVs dc/dVp + drho/dVs dc/drho,
the effective kernel DAzi's consumer forms (CalSurfG_parallel.f90:2367-2374).

Lsen_Gsc is returned as a constant (the first-order azimuthal term is linear
in Gc/Gs with Lsen evaluated on the isotropic model, FwdAzimuthalAniMap.f90
:43-56); `azimuthal_phase_velocity` forms
    c(psi) = c0 + sum_j Lsen_j (Gc_j cos 2 psi + Gs_j sin 2 psi),
differentiable in c0 (hence in Vs) and in Gc, Gs.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


def _i64(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a, np.int64), device=dev)


class ColumnBatch:
    """Structure of a ragged batch on the device: per column its node
    depths (CSR node_off, depz) and ascending periods (CSR per_off,
    periods), and minthk.  The node velocities are the differentiable
    input of `phase_velocity`."""

    def __init__(self, node_off, depz, per_off, periods, minthk, device="cuda"):
        dev = torch.device(device)
        node_off = np.ascontiguousarray(node_off, np.int64)
        per_off = np.ascontiguousarray(per_off, np.int64)
        nz = np.diff(node_off)
        K = np.diff(per_off)
        sen_off = np.concatenate([[0], np.cumsum(K * nz)]).astype(np.int64)
        ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))]).astype(np.int64)
        self.device = dev
        self.ncols = node_off.size - 1
        self.minthk = float(minthk)
        self.nnodes = int(node_off[-1])
        self.nper = int(per_off[-1])
        self.nsen = int(sen_off[-1])
        self.nls = int(ls_off[-1])
        self.node_off = _i64(node_off, dev)
        self.per_off = _i64(per_off, dev)
        self.sen_off = _i64(sen_off, dev)
        self.ls_off = _i64(ls_off, dev)
        self.depz = torch.as_tensor(np.ascontiguousarray(depz, np.float32), device=dev)
        self.periods = torch.as_tensor(np.ascontiguousarray(periods, np.float64), device=dev)
        # gather indices of the kernel entries: entry e = sen_off[c] + k + K_c i
        # belongs to period per_off[c] + k and node node_off[c] + i
        col = np.repeat(np.arange(self.ncols), K * nz)
        local = np.arange(self.nsen) - sen_off[col]
        k = local % K[col]
        i = local // K[col]
        self._sen_period = _i64(per_off[col] + k, dev)
        self._sen_node = _i64(node_off[col] + i, dev)
        colp = np.repeat(np.arange(self.ncols), K * (nz - 1))
        localp = np.arange(self.nls) - ls_off[colp]
        self._ls_period = _i64(per_off[colp] + localp % K[colp], dev)
        self._ls_interval = _i64(node_off[colp] - colp + localp // K[colp], dev)
        self.nintervals = int(self.nnodes - self.ncols)

    @classmethod
    def from_grid(cls, nx, ny, depz, periods, minthk, device="cuda"):
        """The regular grid of the reference's interface (every column the
        same depth grid and periods), columns in the order post = ii +
        (jj-1) nx."""
        n = nx * ny
        nz = len(depz)
        K = len(periods)
        return cls(np.arange(n + 1) * nz, np.tile(np.asarray(depz, np.float32), n),
                   np.arange(n + 1) * K, np.tile(np.asarray(periods, np.float64), n), minthk,
                   device)

    def run(self, vs, vp=None, rho=None, lsen=True, flags=0):
        """Forward call of the library on the current stream (no autograd).
        flags: FORM_LOVE / FORM_GROUP (then lsen=False).
        Returns pv, (sen_vs, sen_vp, sen_rho), lsen, status."""
        L = _lib.load()
        dev = self.device
        vs = vs.detach().to(dev, torch.float32).contiguous()
        if vp is not None:
            vp = vp.detach().to(dev, torch.float32).contiguous()
            rho = rho.detach().to(dev, torch.float32).contiguous()
        pv = torch.empty(self.nper, dtype=torch.float64, device=dev)
        sen = [torch.empty(self.nsen, dtype=torch.float64, device=dev) for _ in range(3)]
        ls = torch.empty(self.nls, dtype=torch.float32, device=dev) if lsen else None
        status = torch.empty(self.ncols, dtype=torch.int32, device=dev)
        P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = L.dazi_dk_batch_dev(self.ncols, P(self.node_off), P(self.depz), P(vs), P(vp),
                                 P(rho), P(self.per_off), P(self.periods),
                                 ctypes.c_float(self.minthk), P(pv), P(self.sen_off), P(sen[0]),
                                 P(sen[1]), P(sen[2]), P(self.ls_off) if lsen else None, P(ls),
                                 _lib.FORM_ADJOINT | flags, P(status), ctypes.c_void_p(stream))
        _lib.check(rc)
        return pv, sen, ls, status

    def vjp(self, grad_pv, kernel):
        """sum_k grad_pv[period] * kernel[entry] onto the nodes."""
        contrib = grad_pv.to(torch.float64)[self._sen_period] * kernel
        out = torch.zeros(self.nnodes, dtype=torch.float64, device=self.device)
        return out.index_add_(0, self._sen_node, contrib)

    def lsen_dense_terms(self, lsen):
        """(period index, interval index) of every Lsen entry, for epilogues."""
        return self._ls_period, self._ls_interval


def brocher_derivatives(vs):
    """dVp/dVs and drho/dVs of the Brocher relations at vs (float64)."""
    v = vs.to(torch.float64)
    vp = 0.9409 + v * (2.0947 + v * (-0.8206 + v * (0.2683 + v * -0.0251)))
    dvp = 2.0947 + v * (2.0 * -0.8206 + v * (3.0 * 0.2683 + v * 4.0 * -0.0251))
    drho_dvp = 1.6612 + vp * (2.0 * -0.4721 + vp * (3.0 * 0.0671 + vp * (4.0 * -0.0043
                                                                          + vp * 5.0 * 0.000106)))
    return dvp, drho_dvp * dvp


class _PhaseVelocity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vs, vp, rho, batch: ColumnBatch, flags: int):
        pv, sen, ls, status = batch.run(vs, vp, rho, lsen=flags == 0, flags=flags)
        if ls is None:
            ls = torch.empty(0, dtype=torch.float32, device=pv.device)
        ctx.batch = batch
        ctx.explicit = vp is not None
        if ctx.explicit:
            ctx.save_for_backward(*sen)
        else:
            dvp, drho = brocher_derivatives(vs.detach())
            k_tot = sen[0] + dvp[batch._sen_node] * sen[1] + drho[batch._sen_node] * sen[2]
            ctx.save_for_backward(k_tot)
        ctx.mark_non_differentiable(ls, status)
        return pv, ls, status

    @staticmethod
    def backward(ctx, grad_pv, grad_ls, grad_status):
        b = ctx.batch
        if ctx.explicit:
            s_vs, s_vp, s_rho = ctx.saved_tensors
            g = [b.vjp(grad_pv, s).to(torch.float32) for s in (s_vs, s_vp, s_rho)]
            return g[0], g[1], g[2], None, None
        (k_tot,) = ctx.saved_tensors
        return b.vjp(grad_pv, k_tot).to(torch.float32), None, None, None, None


def phase_velocity(vs, batch: ColumnBatch, vp=None, rho=None):
    """Rayleigh phase velocity of every (column, period) of the batch and
    the Gc/Gs kernel, differentiable in vs (and vp, rho when given).
    Returns (c [nper] float64, lsen [nls] float32, status [ncols] int32)."""
    if (vp is None) != (rho is None):
        raise ValueError("vp and rho must be given together")
    return _PhaseVelocity.apply(vs, vp, rho, batch, 0)


def dispersion_velocity(vs, batch: ColumnBatch, vp=None, rho=None, iwave=2, igr=0):
    """Love (iwave = 1) or Rayleigh (iwave = 2) phase (igr = 0) or group
    (igr > 0) velocity of every (column, period), as surfdisp96 takes
    iwave/igr, differentiable in vs (and vp, rho when given).  Group
    velocity is the reference's quotient of the phase roots at t/(1+h) and
    t/(1-h); its gradient is the exact derivative of that quotient.  No
    Gc/Gs kernel (a Rayleigh phase kernel: `phase_velocity`).
    Returns (c [nper] float64, status [ncols] int32)."""
    if (vp is None) != (rho is None):
        raise ValueError("vp and rho must be given together")
    if iwave not in (1, 2):
        raise ValueError(f"iwave must be 1 (Love) or 2 (Rayleigh), got {iwave}")
    flags = (_lib.FORM_LOVE if iwave == 1 else 0) | (_lib.FORM_GROUP if igr > 0 else 0)
    c, _, status = _PhaseVelocity.apply(vs, vp, rho, batch, flags)
    return c, status


def azimuthal_phase_velocity(c0, lsen, gc, gs, psi, batch: ColumnBatch):
    """c(psi) = c0 + sum_j Lsen_j (Gc_j cos 2 psi + Gs_j sin 2 psi) per
    (column, period): gc, gs per depth interval (batch.nintervals, the
    nz_c - 1 intervals of every column in order), psi per (column, period)."""
    per_i, int_i = batch.lsen_dense_terms(lsen)
    c2 = torch.cos(2.0 * psi.to(torch.float64))
    s2 = torch.sin(2.0 * psi.to(torch.float64))
    term = lsen.to(torch.float64) * (gc.to(torch.float64)[int_i] * c2[per_i]
                                     + gs.to(torch.float64)[int_i] * s2[per_i])
    return c0 + torch.zeros_like(c0).index_add(0, per_i, term)
