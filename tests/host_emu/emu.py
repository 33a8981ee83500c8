"""Loader of the host build of the library's device code (test
infrastructure: checks the device arithmetic against the oracle on CPU)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
        _lib = ctypes.CDLL(os.path.join(HERE, "_build", "libemu.so"))
    return _lib


def ti_batch(node_off, depz, vs, per_off, periods, minthk, pv):
    """Lsen_Gsc of a ragged batch (dazi_dk_batch layout) from the given
    phase velocities, computed by the device code built for the host."""
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    nz = np.diff(node_off)
    K = np.diff(per_off)
    ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))]).astype(np.int64)
    ls = np.zeros(max(int(ls_off[-1]), 1), np.float32)
    i64, f32, f64 = ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    rc = lib().emu_ti_batch(i64(node_off.size - 1), P(node_off, i64),
                            P(np.ascontiguousarray(depz, np.float32), f32),
                            P(np.ascontiguousarray(vs, np.float32), f32), P(per_off, i64),
                            P(np.ascontiguousarray(periods, np.float64), f64), f32(minthk),
                            P(np.ascontiguousarray(pv, np.float64), f64), P(ls_off, i64),
                            P(ls, f32))
    return rc, ls, ls_off


def root_batch(node_off, depz, vs, per_off, periods, minthk, scan32=True, ifunc=2, group=False,
               fast=False):
    """pv (sngl(c) as the library writes it; the group velocity when
    group), status and the number of secular evaluations of the root search
    of a ragged batch; ifunc 1 Love, 2 Rayleigh; fast the Brent refinement."""
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    pv = np.zeros(max(int(per_off[-1]), 1))
    st = np.zeros(max(node_off.size - 1, 1), np.int32)
    ev = ctypes.c_longlong(0)
    i64, f32, f64 = ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    rc = lib().emu_root_batch(i64(node_off.size - 1), P(node_off, i64),
                              P(np.ascontiguousarray(depz, np.float32), f32),
                              P(np.ascontiguousarray(vs, np.float32), f32), P(per_off, i64),
                              P(np.ascontiguousarray(periods, np.float64), f64), f32(minthk),
                              int(scan32), int(ifunc), int(bool(group)), int(bool(fast)),
                              P(pv, f64),
                              P(st, ctypes.c_int), ctypes.byref(ev))
    return rc, pv, st, ev.value


def adjoint_batch(node_off, depz, vs, per_off, periods, minthk, ifunc=2, group=False,
                  drop_every=0, fast=False):
    """Adjoint form of a ragged batch by the device code built for the host:
    rc, pv, status, (sen_vs, sen_vp, sen_rho) in the batch layout, sen_off,
    and the mask of (column, period) entries whose root at t1b was set to 0
    (drop_every > 0, group only: the planted group fallback)."""
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    nz = np.diff(node_off)
    K = np.diff(per_off)
    sen_off = np.concatenate([[0], np.cumsum(K * nz)]).astype(np.int64)
    npv = max(int(per_off[-1]), 1)
    pv = np.zeros(npv)
    st = np.zeros(max(node_off.size - 1, 1), np.int32)
    sen = [np.zeros(max(int(sen_off[-1]), 1)) for _ in range(3)]
    dropped = np.zeros(npv, np.uint8)
    i64, f32, f64 = ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    rc = lib().emu_adjoint_batch(i64(node_off.size - 1), P(node_off, i64),
                                 P(np.ascontiguousarray(depz, np.float32), f32),
                                 P(np.ascontiguousarray(vs, np.float32), f32), P(per_off, i64),
                                 P(np.ascontiguousarray(periods, np.float64), f64), f32(minthk),
                                 int(ifunc), int(bool(group)), int(drop_every),
                                 int(bool(fast)), P(pv, f64),
                                 P(st, ctypes.c_int), P(sen_off, i64), P(sen[0], f64),
                                 P(sen[1], f64), P(sen[2], f64), P(dropped, ctypes.c_ubyte))
    return rc, pv, st, sen, sen_off, dropped.astype(bool)


def fmm_batch(params, pv, inst_period, scx, scz, rc_off, rcx, rcz, fields=False):
    """Receiver times (and, when fields, the coarse fields (ninst, nnx, nnz))
    of the library's traveltime device code built for the host; params is a
    ctypes structure with dazi_fmm_params' layout."""
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    pv = np.asfortranarray(pv, np.float64)
    ninst = len(inst_period)
    rc_off = np.ascontiguousarray(rc_off, np.int64)
    times = np.zeros(max(int(rc_off[-1]), 1), np.float32)
    nnx, nnz = (params.nx - 3) * params.gdx + 1, (params.ny - 3) * params.gdz + 1
    ttn = np.zeros((ninst, nnx, nnz), np.float32) if fields else None
    code = ctypes.c_int(0)
    f32, i32 = ctypes.c_float, ctypes.c_int
    rc = lib().emu_fmm_batch(ctypes.byref(params), P(pv, ctypes.c_double), int(pv.shape[1]), ninst,
                             P(np.ascontiguousarray(inst_period, np.int32), i32),
                             P(np.ascontiguousarray(scx, np.float32), f32),
                             P(np.ascontiguousarray(scz, np.float32), f32), P(rc_off, ctypes.c_longlong),
                             P(np.ascontiguousarray(rcx, np.float32), f32),
                             P(np.ascontiguousarray(rcz, np.float32), f32), P(times, f32),
                             None if ttn is None else P(ttn, f32), ctypes.byref(code))
    if rc:
        raise RuntimeError(f"emu fmm_batch: {rc} (instance error {code.value})")
    return (times[:int(rc_off[-1])], ttn) if fields else times[:int(rc_off[-1])]
