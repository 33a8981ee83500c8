"""LSMR on the GPU over the G-row triplets (dazi_lsmr_dev in
include/dazi_dk.h): the least-squares solve the depth kernels feed,
mirroring the reference's LSMR call (code/src_inv_iso_joint/lsmrModule.f90:36)
and its SciPy backend (code/depthkernel_lab/scipy_lsmr_triplet_solver.py)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib


@dataclass
class LsmrResult:
    x: torch.Tensor          # (n,) float64 on the device
    istop: int
    itn: int
    normA: float
    condA: float
    normr: float
    normAr: float
    normx: float


def lsmr(row, col, val, b, m: int, n: int, *, damp=0.0, atol=1e-6, btol=1e-6, conlim=1e8,
         maxiter=None, index_base=1, stream=None) -> LsmrResult:
    """Solve min ||(A; damp I) x - (b; 0)|| for the sparse A given by the
    triplets (row, col, val): device tensors int32, int32, float32 (the
    reference's iw/rw layout), b float64 (m,).  maxiter defaults to
    min(m, n), as scipy.sparse.linalg.lsmr's."""
    L = _lib.load()
    dev = b.device
    if maxiter is None:
        maxiter = min(m, n)
    x = torch.empty(n, dtype=torch.float64, device=dev)
    istop, itn = ctypes.c_int(0), ctypes.c_int(0)
    norms = (ctypes.c_double * 5)()
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    _lib.check(L.dazi_lsmr_dev(int(m), int(n), int(val.numel()), P(row), P(col), P(val),
                               int(index_base), P(b), float(damp), float(atol), float(btol),
                               float(conlim), int(maxiter), P(x), ctypes.byref(istop),
                               ctypes.byref(itn), norms, ctypes.c_void_p(s)))
    return LsmrResult(x, istop.value, itn.value, *list(norms))
