"""Azimuthal phase-velocity maps on the GPU (dazi_dk_azimuthal_map_dev),
the computation of FwdAzimuthalAniMap.f90:43-86; formats.write_azimuthal_map
writes them in the reference's layout."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


def azimuthal_map(Lsen_Gsc, gcf, gsf, tRcV, device="cuda"):
    """Lsen_Gsc (nx*ny, K, nz-1), gcf/gsf (nx-2, ny-2, nz-1), tRcV
    ((nx-2)*(ny-2), K).  Returns cos, sin, amp, amp_rel, angle, each
    ((nx-2)*(ny-2), K) float32."""
    L = _lib.load()
    dev = torch.device(device)
    gcf = np.asarray(gcf)
    nvx, nvz, nzm1 = gcf.shape
    K = np.shape(Lsen_Gsc)[1]
    F = lambda a, dt: torch.as_tensor(np.asarray(a, dt).ravel(order="F"), device=dev)  # noqa: E731
    ls, gc, gs = F(Lsen_Gsc, np.float32), F(gcf, np.float32), F(gsf, np.float32)
    ci = F(tRcV, np.float64)
    out = [torch.empty(nvx * nvz * K, dtype=torch.float32, device=dev) for _ in range(5)]
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.dazi_dk_azimuthal_map_dev(nvx + 2, nvz + 2, nzm1 + 1, K, P(ls), P(gc), P(gs), P(ci),
                                     *[P(o) for o in out],
                                     ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    _lib.check(rc)
    torch.cuda.synchronize(dev)
    return tuple(o.cpu().numpy().reshape((nvx * nvz, K), order="F") for o in out)
