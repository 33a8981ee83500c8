"""G rows of the LSMR system from the depth kernels (dazi_dk_grows_dev):
the consumer of the stage (CalSurfG_parallel.f90:2363-2400), on the GPU.

    rw, iw, col, nnz = g_rows(vels, sen_vs, sen_vp, sen_rho, lsen, ray_period, ray_id,
                              cell_off, cell, fdm, fdmc, fdms)

vels (nvx+2, nvz+2, nz) float32 and the kernels in the reference's layouts
(sen_* (nxy, K, nz) float64, lsen (nxy, K, nz-1) float32 or None); rays in
CSR with ascending cell indices (jj-1)*nvx + kk-1 and their path weights.
Returns the sparse entries in the reference's order and the count per ray.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


def g_rows(vels, sen_vs, sen_vp, sen_rho, lsen, ray_period, ray_id, cell_off, cell, fdm,
           fdmc=None, fdms=None, ftol=1e-4, cap=None, device="cuda"):
    L = _lib.load()
    dev = torch.device(device)
    nxv, nzv, nz = np.shape(vels)
    nvx, nvz = nxv - 2, nzv - 2
    K = np.shape(sen_vs)[1]
    F = lambda a, dt: torch.as_tensor(np.asarray(a, dt).ravel(order="F"), device=dev)  # noqa: E731
    C = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dt), device=dev)  # noqa: E731
    d_vels = F(vels, np.float32)
    d_s = [F(x, np.float64) for x in (sen_vs, sen_vp, sen_rho)]
    d_ls = None if lsen is None else F(lsen, np.float32)
    d_per, d_id = C(ray_period, np.int32), C(ray_id, np.int32)
    d_off, d_cell = C(cell_off, np.int64), C(cell, np.int32)
    d_fdm = C(fdm, np.float32)
    d_fc = None if fdmc is None else C(fdmc, np.float32)
    d_fs = None if fdms is None else C(fdms, np.float32)
    nrays = int(np.size(cell_off)) - 1
    if cap is None:
        cap = int(np.asarray(cell_off)[-1]) * (nz - 1) * (3 if lsen is not None else 1)
    cap = max(int(cap), 1)
    rw = torch.empty(cap, dtype=torch.float32, device=dev)
    iw = torch.empty(cap, dtype=torch.int32, device=dev)
    col = torch.empty(cap, dtype=torch.int32, device=dev)
    nnz = torch.zeros(max(nrays, 1), dtype=torch.int64, device=dev)
    tot = ctypes.c_longlong(0)
    P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.dazi_dk_grows_dev(nvx, nvz, nz, K, P(d_vels), P(d_s[0]), P(d_s[1]), P(d_s[2]), P(d_ls),
                             nrays, P(d_per), P(d_id), P(d_off), P(d_cell), P(d_fdm), P(d_fc),
                             P(d_fs), ctypes.c_float(ftol), cap, P(rw), P(iw), P(col), P(nnz),
                             ctypes.byref(tot), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    _lib.check(rc)
    torch.cuda.synchronize(dev)
    n = tot.value
    return (rw[:n].cpu().numpy(), iw[:n].cpu().numpy(), col[:n].cpu().numpy(),
            nnz[:nrays].cpu().numpy())
