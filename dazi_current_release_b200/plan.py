"""Plans: an uneven-column batch bound once to device tensors and run many
times as one CUDA-graph launch (dazi_dk_plan_* in include/dazi_dk.h).

    p = BatchPlan(node_off, depz, vs, per_off, periods, minthk)   # builds, tunes, captures
    p.run()            # recompute from the current contents of p.vs (in place)
    p.pv, p.sen_vs, ..., p.lsen, p.status                         # bound outputs

The structure (node depths, periods) is fixed at creation; the velocities
may change between runs (write into p.vs).  The autotuner's choice is in
p.config().  fast_root=True refines each period's bracket by Brent's method
(DAZI_FORM_FAST_ROOT) instead of the reference's nevill(); full_stack=True
runs the adjoint and Gc/Gs sweeps without the depth cut
(DAZI_FORM_FULL_STACK).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .batch import output_offsets


class BatchPlan:
    def __init__(self, node_off, depz, vs, per_off, periods, minthk, *, vp=None, rho=None,
                 kernels=True, lsen=True, tune=True, scan32=False, fast_root=False,
                 full_stack=False, device="cuda"):
        dev = torch.device(device)
        self.L = _lib.load()
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)  # noqa: E731
        node_off = np.ascontiguousarray(node_off, np.int64)
        per_off = np.ascontiguousarray(per_off, np.int64)
        sen_off, ls_off = output_offsets(node_off, per_off)
        self.ncols = node_off.size - 1
        self.node_off, self.per_off = t(node_off, torch.int64), t(per_off, torch.int64)
        self.sen_off, self.ls_off = t(sen_off, torch.int64), t(ls_off, torch.int64)
        self.depz = t(depz, torch.float32)
        self.periods = t(periods, torch.float64)
        self.vs = t(vs, torch.float32)
        self.vp = None if vp is None else t(vp, torch.float32)
        self.rho = None if rho is None else t(rho, torch.float32)
        self.pv = torch.zeros(int(per_off[-1]), dtype=torch.float64, device=dev)
        z = lambda n, dt: torch.zeros(n, dtype=dt, device=dev)  # noqa: E731
        ns, nl = int(sen_off[-1]), int(ls_off[-1])
        self.sen_vs, self.sen_vp, self.sen_rho = ((z(ns, torch.float64) for _ in range(3))
                                                  if kernels else (None, None, None))
        self.lsen = z(nl, torch.float32) if lsen else None
        self.status = z(self.ncols, torch.int32)
        P = lambda x: None if x is None else ctypes.c_void_p(x.data_ptr())  # noqa: E731
        form = (_lib.FORM_ADJOINT | (_lib.FORM_SCAN_FP32 if scan32 else 0) |
                (_lib.FORM_FAST_ROOT if fast_root else 0) |
                (_lib.FORM_FULL_STACK if full_stack else 0))
        h = ctypes.c_void_p(None)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = self.L.dazi_dk_plan_create(
            self.ncols, P(self.node_off), P(self.depz), P(self.vs), P(self.vp), P(self.rho),
            P(self.per_off), P(self.periods), ctypes.c_float(minthk), P(self.pv),
            P(self.sen_off) if kernels else None, P(self.sen_vs), P(self.sen_vp), P(self.sen_rho),
            P(self.ls_off) if lsen else None, P(self.lsen), form, P(self.status), int(tune),
            ctypes.c_void_p(stream), ctypes.byref(h))
        _lib.check(rc)
        self.handle = h

    def run(self, stream=None):
        """One graph launch on the current (or given) stream."""
        s = stream if stream is not None else torch.cuda.current_stream(self.vs.device).cuda_stream
        _lib.check(self.L.dazi_dk_plan_launch(self.handle, ctypes.c_void_p(s)))

    def status_check(self):
        """DaziError if the last completed run produced a non-finite Lsen."""
        _lib.check(self.L.dazi_dk_plan_status(self.handle))

    def config(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = (ctypes.c_float * 3)()
        _lib.check(self.L.dazi_dk_plan_config(self.handle, ctypes.byref(a), ctypes.byref(b),
                                              ctypes.byref(c), ms))
        return {"root_block": a.value // 100, "root_blocks_per_sm": a.value % 100,
                "adjoint_blocks_per_sm": b.value,
                "ti_blocks_per_sm": c.value, "tuned_ms": list(ms)}

    def close(self):
        if self.handle:
            self.L.dazi_dk_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
