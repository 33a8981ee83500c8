"""Ragged batch interface: columns with their own depth grids and period
lists (CSR layout), e.g. the Voronoi-cell columns of many realisations.

This replaces the reference's fixed column tiles (pdsurf_tile_columns /
ti_tile_columns, code/depthkernel_lab/depthkernel_ti_process_batch.py:17-28,
pdsurf_tile_senk_solver.py:184-245): the library sorts the columns into
32-column tiles by layer and period count and runs each kernel as one launch.
Per-column outputs keep the reference's per-column layouts: pv(K_c),
sen_*(K_c, nz_c) and Lsen_Gsc(K_c, nz_c - 1), column-major.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def output_offsets(node_off, per_off):
    """CSR offsets of the kernel (K_c * nz_c) and Lsen (K_c * (nz_c - 1))
    outputs of every column."""
    nz = np.diff(node_off)
    K = np.diff(per_off)
    sen_off = np.concatenate([[0], np.cumsum(K * nz)]).astype(np.int64)
    ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))]).astype(np.int64)
    return sen_off, ls_off


class BatchResult(dict):
    def column(self, c):
        """Per-column views: (pv[K], sen_vs[K, nz], sen_vp, sen_rho, lsen[K, nz-1])."""
        p0, p1 = self["per_off"][c], self["per_off"][c + 1]
        K = p1 - p0
        out = [self["pv"][p0:p1]]
        if self.get("sen_vs") is not None:
            s0, s1 = self["sen_off"][c], self["sen_off"][c + 1]
            nz = (s1 - s0) // K
            for n in ("sen_vs", "sen_vp", "sen_rho"):
                out.append(self[n][s0:s1].reshape((K, nz), order="F"))
        if self.get("lsen") is not None:
            l0, l1 = self["ls_off"][c], self["ls_off"][c + 1]
            out.append(self["lsen"][l0:l1].reshape((K, (l1 - l0) // K), order="F"))
        return tuple(out)


def depthkernel_batch(node_off, depz, vs, per_off, periods, minthk, *, vp=None, rho=None,
                      form=_lib.FORM_ADJOINT, kernels=True, lsen=True) -> BatchResult:
    """Run the stage on a ragged batch through the host C-ABI entry
    dazi_dk_batch.  form: FORM_PLAIN or FORM_ADJOINT, optionally OR-ed with
    FORM_LOVE / FORM_GROUP (then lsen=False: Lsen_Gsc is a Rayleigh phase
    kernel) or, for Rayleigh phase velocity, FORM_SCAN_FP32, and
    FORM_FULL_STACK (the adjoint and Lsen_Gsc sweeps without the depth
    cut).  Raises
    DaziError for errors; status (per column) holds the first period without
    a root (0 when all have one)."""
    L = _lib.load()
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    depz = np.ascontiguousarray(depz, np.float32)
    vs = np.ascontiguousarray(vs, np.float32)
    periods = np.ascontiguousarray(periods, np.float64)
    if vp is not None:
        vp = np.ascontiguousarray(vp, np.float32)
        rho = np.ascontiguousarray(rho, np.float32)
    ncols = node_off.size - 1
    sen_off, ls_off = output_offsets(node_off, per_off)
    pv = np.zeros(int(per_off[-1]), np.float64)
    sen = [np.zeros(int(sen_off[-1]), np.float64) for _ in range(3)] if kernels else [None] * 3
    ls = np.zeros(int(ls_off[-1]), np.float32) if lsen else None
    status = np.zeros(ncols, np.int32)
    P = lambda a, t: None if a is None else a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    i64, f32, f64 = ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    rc = L.dazi_dk_batch(ncols, P(node_off, i64), P(depz, f32), P(vs, f32), P(vp, f32),
                         P(rho, f32), P(per_off, i64), P(periods, f64), ctypes.c_float(minthk),
                         P(pv, f64), P(sen_off, i64) if kernels else None, P(sen[0], f64),
                         P(sen[1], f64), P(sen[2], f64), P(ls_off, i64) if lsen else None,
                         P(ls, f32), int(form), P(status, ctypes.c_int))
    _lib.check(rc)
    return BatchResult(pv=pv, sen_vs=sen[0], sen_vp=sen[1], sen_rho=sen[2], lsen=ls,
                       status=status, node_off=node_off, per_off=per_off, sen_off=sen_off,
                       ls_off=ls_off, rc=rc)
