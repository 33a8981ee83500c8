"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates the reference Fortran depth-kernel stage in C
(oracle/dk_oracle.c, oracle/tregn_oracle.c).  Only the tests, the smoke check
and bench.py's CPU-baseline leg import this module, and only as the checker or
the timed CPU baseline; the shipped library never calls it.

Array conventions follow the reference Fortran interfaces
(code/src_inv_iso_joint/CalSurfG.f90:1-15 and depthkernelTI.f90:2-14):
``vel`` is (nx, ny, nz) in Fortran order, outputs are (nx*ny, kmax[, nz]) in
Fortran order.  numpy arrays passed here use ``order="F"``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_dk.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_long)


def build() -> str:
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class FmmParams(ctypes.Structure):
    """OrFmmParams (dk_oracle.h): the model grid and the traveltime solver's
    settings, defaults as CalSurfG_parallel.f90:1900-1911 sets them."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("goxd", ctypes.c_float),
                ("gozd", ctypes.c_float), ("dvxd", ctypes.c_float), ("dvzd", ctypes.c_float),
                ("gdx", ctypes.c_int), ("gdz", ctypes.c_int), ("asgr", ctypes.c_int),
                ("sgdl", ctypes.c_int), ("sgs", ctypes.c_int), ("fom", ctypes.c_int),
                ("snb", ctypes.c_float), ("earth", ctypes.c_float)]


def fmm_params(nx, ny, goxd, gozd, dvxd, dvzd, gdx=5, gdz=5, asgr=1, sgdl=8, sgs=8, fom=1,
               snb=0.5, earth=6371.0):
    return FmmParams(nx, ny, goxd, gozd, dvxd, dvzd, gdx, gdz, asgr, sgdl, sgs, fom, snb, earth)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.or_brocher.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p]
        L.or_brocher.restype = None
        L.or_refine.argtypes = [ctypes.c_float, ctypes.c_int, _f32p, _f32p, _f32p, _f32p,
                                _f32p, _f32p, _f32p, _f32p, _i32p]
        L.or_refine.restype = ctypes.c_int
        L.or_surfdisp96_ex.argtypes = [_f32p, _f32p, _f32p, _f32p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       _f64p, _f64p, ctypes.c_double, ctypes.c_int, _i32p]
        L.or_surfdisp96_ex.restype = ctypes.c_int
        L.or_depthkernel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p,
                                     _f64p, _f64p, _f64p, _f64p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, _f64p, _f32p, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_float, _i32p, _i64p]
        L.or_depthkernel.restype = ctypes.c_int
        L.or_phase.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p,
                               _f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p, _f32p,
                               ctypes.c_float, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                               _i32p, _i32p]
        L.or_phase.restype = ctypes.c_int
        if hasattr(L, "or_depthkernelTI"):
            L.or_depthkernelTI.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p,
                                           _f32p, _f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           _f64p, _f32p, ctypes.c_float, _f32p, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, _i32p]
            L.or_depthkernelTI.restype = ctypes.c_int
            L.or_tregn96.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                     _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                     ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p]
            L.or_tregn96.restype = ctypes.c_int
            L.or_tregn96_ex.argtypes = L.or_tregn96.argtypes + [ctypes.c_int, ctypes.c_int, _f64p]
            L.or_tregn96_ex.restype = ctypes.c_int
            L.or_tregn96_cd.argtypes = L.or_tregn96.argtypes[:16] + [_f64p] + \
                L.or_tregn96.argtypes[17:] + [ctypes.c_int, ctypes.c_int, _f64p]
            L.or_tregn96_cd.restype = ctypes.c_int
            d7 = [ctypes.c_int] + [_f64p] * 7
            L.or_ti_secular_d.argtypes = d7 + [ctypes.c_double, ctypes.c_double]
            L.or_ti_secular_d.restype = ctypes.c_double
            L.or_ti_root_d.argtypes = d7 + [ctypes.c_double] * 3 + [_f64p]
            L.or_ti_root_d.restype = ctypes.c_int
            L.or_ti_root_fd.argtypes = d7 + [ctypes.c_double] * 4 + [ctypes.c_int, _i32p, _i32p,
                                                                      _i32p, _f64p, ctypes.c_int]
            L.or_ti_root_fd.restype = ctypes.c_int
        L.or_surfdisp96_split.argtypes = [_f32p] * 4 + [ctypes.c_int] * 2 + [_f64p, _f64p, _i32p,
                                                                             _i32p]
        L.or_surfdisp96_split.restype = ctypes.c_int
        L.or_surfdisp96_d.argtypes = [_f64p, _f64p, _f64p, _f64p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _f64p, _f64p, ctypes.c_double]
        L.or_surfdisp96_d.restype = ctypes.c_int
        L.or_batch.argtypes = [ctypes.c_long, _i64p, _f32p, _f32p, _i64p, _f64p, ctypes.c_float,
                               _f64p, _i64p, _f64p, _f64p, _f64p, _i64p, _f32p, ctypes.c_int]
        L.or_batch.restype = ctypes.c_int
        L.or_batch_ti.argtypes = [ctypes.c_long, _i64p, _f32p, _f32p, _i64p, _f64p,
                                  ctypes.c_float, _f64p, ctypes.c_double, _f64p, _i64p, _f32p,
                                  ctypes.c_int]
        L.or_batch_ti.restype = ctypes.c_int
        L.or_batch_fd.argtypes = [ctypes.c_long, _i64p, _f32p, _f32p, _i64p, _f64p,
                                  ctypes.c_float, _f64p, _i64p, _f64p, _f64p, _f64p, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_float, _i32p, ctypes.c_int]
        L.or_batch_fd.restype = ctypes.c_int
        L.or_grows.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f64p,
                               _f64p, _f64p, _f32p, ctypes.c_long, _i32p, _i32p, _i64p, _i32p,
                               _f32p, _f32p, _f32p, ctypes.c_float, ctypes.c_long, _f32p, _i32p,
                               _i32p, _i64p]
        L.or_grows.restype = ctypes.c_long
        L.or_azimap.argtypes = [ctypes.c_int] * 4 + [_f32p] * 3 + [_f64p] + [_f32p] * 5
        L.or_azimap.restype = None
        L.or_fmm_batch.argtypes = [ctypes.POINTER(FmmParams), _f64p, ctypes.c_int, _i32p, _f32p,
                                   _f32p, _i64p, _f32p, _f32p, _f32p, _f32p, ctypes.c_int]
        L.or_fmm_batch.restype = ctypes.c_int
        L.or_fmm_travel.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 5 + \
            [ctypes.c_int, ctypes.c_float, _f32p, ctypes.c_float, ctypes.c_float, _f32p, _i32p]
        L.or_fmm_travel.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(ct)


def brocher(vs):
    vs = np.ascontiguousarray(vs, dtype=np.float32)
    vp = np.empty_like(vs)
    rho = np.empty_like(vs)
    lib().or_brocher(vs.size, _p(vs, _f32p), _p(vp, _f32p), _p(rho, _f32p))
    return vp, rho


def refine(minthk, dep, vp, vs, rho):
    """Grid-to-layer refinement; returns (rthk, rvp, rvs, rrho, nsublay)."""
    dep = np.ascontiguousarray(dep, np.float32)
    vp = np.ascontiguousarray(vp, np.float32)
    vs = np.ascontiguousarray(vs, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    out = [np.zeros(200, np.float32) for _ in range(4)]
    ns = np.zeros(200, np.int32)
    r = lib().or_refine(ctypes.c_float(minthk), dep.size, _p(dep, _f32p), _p(vp, _f32p),
                        _p(vs, _f32p), _p(rho, _f32p), *[_p(o, _f32p) for o in out],
                        _p(ns, _i32p))
    if r < 0:
        raise ValueError("refined layer count exceeds 200")
    return tuple(o[:r].copy() for o in out) + (ns[: dep.size - 1].copy(),)


def surfdisp96(thk, vp, vs, rho, periods, iwave=2, igr=0, mode=1, iflsph=1,
               tol=1e-6, round_f32=True):
    """Returns (cg[kmax], status, evals[kmax])."""
    thk = np.ascontiguousarray(thk, np.float32)
    vp = np.ascontiguousarray(vp, np.float32)
    vs = np.ascontiguousarray(vs, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    t = np.ascontiguousarray(periods, np.float64)
    cg = np.zeros(t.size, np.float64)
    ev = np.zeros(t.size, np.int32)
    st = lib().or_surfdisp96_ex(_p(thk, _f32p), _p(vp, _f32p), _p(vs, _f32p), _p(rho, _f32p),
                                thk.size, iflsph, iwave, mode, igr, t.size, _p(t, _f64p),
                                _p(cg, _f64p), tol, int(round_f32), _p(ev, _i32p))
    return cg, st, ev


def surfdisp96_split(thk, vp, vs, rho, periods):
    """Rayleigh phase velocity (reference arithmetic) with the secular
    evaluations of every period split: returns (cg, status, evals, scan)
    where scan counts getsol's bracket scan and evals - scan nevill's."""
    f = lambda x: np.ascontiguousarray(x, np.float32)  # noqa: E731
    t = np.ascontiguousarray(periods, np.float64)
    cg = np.zeros(t.size)
    ev = np.zeros(t.size, np.int32)
    sc = np.zeros(t.size, np.int32)
    st = lib().or_surfdisp96_split(*[_p(f(x), _f32p) for x in (thk, vp, vs, rho)], len(thk),
                                   t.size, _p(t, _f64p), _p(cg, _f64p), _p(ev, _i32p),
                                   _p(sc, _i32p))
    return cg, st, ev, sc


def depthkernel(vel, depz, periods, minthk, vp=None, rho=None, iwave=2, igr=0,
                col_start=1, col_count=None, nthreads=0, tol=1e-6, round_f32=True,
                kernels=True, dln=0.01, exact=False):
    """Oracle of ``depthkernel`` (CalSurfG.f90:1-113, default_fortran_fd).

    round_f32=False keeps the roots unrounded; exact=True runs the whole model
    pipeline in double (no real*4 stores) with the exact FD step, which with a
    tight tol and small dln resolves the derivative itself (a checker, not the
    reference's arithmetic).

    Returns dict with pvRc (nxy,K), sen_vs/sen_vp/sen_rho (nxy,K,nz) F-order,
    status (nxy,) and evals (total secular evaluations).
    """
    vel = np.asfortranarray(vel, np.float32)
    nx, ny, nz = vel.shape
    t = np.ascontiguousarray(periods, np.float64)
    K = t.size
    depz = np.ascontiguousarray(depz, np.float32)
    nxy = nx * ny
    if col_count is None:
        col_count = nxy - col_start + 1
    vp_a = None if vp is None else np.asfortranarray(vp, np.float32)
    rho_a = None if rho is None else np.asfortranarray(rho, np.float32)
    pv = np.zeros((nxy, K), np.float64, order="F")
    if kernels:
        svs = np.zeros((nxy, K, nz), np.float64, order="F")
        svp = np.zeros_like(svs)
        srh = np.zeros_like(svs)
    else:
        svs = svp = srh = None
    status = np.zeros(nxy, np.int32)
    ev = ctypes.c_long(0)
    if kernels:
        r = lib().or_depthkernel(nx, ny, nz, _p(vel, _f32p), _p(vp_a, _f32p), _p(rho_a, _f32p),
                                 _p(pv, _f64p), _p(svs, _f64p), _p(svp, _f64p), _p(srh, _f64p),
                                 iwave, igr, K, _p(t, _f64p), _p(depz, _f32p),
                                 ctypes.c_float(minthk), col_start, col_count, nthreads, tol,
                                 2 if exact else (0 if round_f32 else 1), ctypes.c_float(dln),
                                 _p(status, _i32p),
                                 ctypes.byref(ev))
        if r != 0:
            raise RuntimeError(f"oracle depthkernel failed ({r})")
        return dict(pvRc=pv, sen_vs=svs, sen_vp=svp, sen_rho=srh, status=status,
                    evals=ev.value)
    evcp = np.zeros((nxy, K), np.int32, order="F")
    r = lib().or_phase(nx, ny, nz, _p(vel, _f32p), _p(vp_a, _f32p), _p(rho_a, _f32p),
                       _p(pv, _f64p), iwave, igr, K, _p(t, _f64p), _p(depz, _f32p),
                       ctypes.c_float(minthk), nthreads, tol, int(round_f32),
                       _p(evcp, _i32p), _p(status, _i32p))
    if r != 0:
        raise RuntimeError(f"oracle phase failed ({r})")
    return dict(pvRc=pv, status=status, evals_cp=evcp)


def depthkernel_ti(vel, depz, periods, minthk, vp=None, rho=None, iwave=2, igr=0,
                   nthreads=0):
    # (nthreads: OpenMP threads over columns; 0 = all)
    """Oracle of ``depthkernelTI`` (depthkernelTI.f90:2-193).

    Returns dict with pvRc (nxy,K) float64 and Lsen_Gsc (nxy,K,nz-1) float32,
    both F-order, plus status (nxy,).
    """
    vel = np.asfortranarray(vel, np.float32)
    nx, ny, nz = vel.shape
    t = np.ascontiguousarray(periods, np.float64)
    K = t.size
    depz = np.ascontiguousarray(depz, np.float32)
    nxy = nx * ny
    vp_a = None if vp is None else np.asfortranarray(vp, np.float32)
    rho_a = None if rho is None else np.asfortranarray(rho, np.float32)
    pv = np.zeros((nxy, K), np.float64, order="F")
    lsen = np.zeros((nxy, K, nz - 1), np.float32, order="F")
    status = np.zeros(nxy, np.int32)
    r = lib().or_depthkernelTI(nx, ny, nz, _p(vel, _f32p), _p(vp_a, _f32p), _p(rho_a, _f32p),
                               _p(pv, _f64p), iwave, igr, K, _p(t, _f64p), _p(depz, _f32p),
                               ctypes.c_float(minthk), _p(lsen, _f32p), 1, nxy, nthreads,
                               _p(status, _i32p))
    if r != 0:
        raise RuntimeError(f"oracle depthkernelTI failed ({r})")
    return dict(pvRc=pv, Lsen_Gsc=lsen, status=status)


def surfdisp96_d(thk, vp, vs, rho, periods, iflsph=1, tol=1e-13):
    """Exact-model surfdisp96 (double model arrays, unrounded roots): a
    checker for derivatives, not the reference's arithmetic."""
    a = [np.ascontiguousarray(x, np.float64) for x in (thk, vp, vs, rho)]
    t = np.ascontiguousarray(periods, np.float64)
    cg = np.zeros(t.size)
    st = lib().or_surfdisp96_d(*[_p(x, _f64p) for x in a], a[0].size, iflsph, t.size,
                               _p(t, _f64p), _p(cg, _f64p), tol)
    return cg, st


def tregn96(thk, TA, TC, TF, TL, TN, rho, periods, cp, nsph=1, dogam=1, full=False,
            cp_double=False):
    """tregn96 partials (dcdah, dcdbv, dcdn as (K, nl) float32); with
    full=True also the FP64 partials [K, 7, nl] (ah, av, bh, bv, n, r, and
    c after the Q shift in [:, 6, 0]).  cp_double=True evaluates them at the
    double phase velocities cp instead of their real*4 values."""
    nl = len(thk)
    f = lambda x: np.ascontiguousarray(x, np.float32)  # noqa: E731
    arr = [f(thk), f(TA), f(TC), f(TF), f(TL), f(TN), f(rho)]
    qp = np.full(nl, 150.0, np.float32)
    qs = np.full(nl, 50.0, np.float32)
    z = np.zeros(nl, np.float32)
    one = np.ones(nl, np.float32)
    t = f(periods)
    K = t.size
    out = [np.zeros((K, nl), np.float32) for _ in range(3)]
    fb = np.zeros((K, 7, nl)) if full else None
    head = [_p(x, _f32p) for x in arr] + [_p(qp, _f32p), _p(qs, _f32p), _p(z, _f32p),
                                          _p(z, _f32p), _p(one, _f32p), _p(one, _f32p)]
    if cp_double:
        c = np.ascontiguousarray(cp, np.float64)
        r = lib().or_tregn96_cd(nl, *head, K, _p(t, _f32p), _p(c, _f64p),
                                *[_p(o, _f32p) for o in out], int(nsph), int(dogam),
                                _p(fb, _f64p))
    else:
        c = f(cp)
        r = lib().or_tregn96_ex(nl, *head, K, _p(t, _f32p), _p(c, _f32p),
                                *[_p(o, _f32p) for o in out], int(nsph), int(dogam),
                                _p(fb, _f64p))
    if r != 0:
        raise RuntimeError("oracle tregn96 failed")
    return (tuple(out) + (fb,)) if full else tuple(out)


def _d7(thk, TA, TC, TF, TL, TN, rho):
    return [np.ascontiguousarray(x, np.float64) for x in (thk, TA, TC, TF, TL, TN, rho)]


def ti_secular(thk, TA, TC, TF, TL, TN, rho, omega, c):
    """TI Rayleigh secular function (up()'s top compound entry) of a flat
    double-precision model at (omega, c): a checker."""
    a = _d7(thk, TA, TC, TF, TL, TN, rho)
    return lib().or_ti_secular_d(len(a[0]), *[_p(x, _f64p) for x in a], omega, c)


def ti_root(thk, TA, TC, TF, TL, TN, rho, omega, c0, xtol=1e-14):
    """Root of the TI secular function nearest c0 (bracketed, Brent)."""
    a = _d7(thk, TA, TC, TF, TL, TN, rho)
    out = ctypes.c_double(0.0)
    r = lib().or_ti_root_d(len(a[0]), *[_p(x, _f64p) for x in a], omega, c0, xtol * c0,
                           ctypes.byref(out))
    if r != 0:
        raise RuntimeError("no TI root near c0")
    return out.value


def ti_root_fd(thk, TA, TC, TF, TL, TN, rho, omega, c0, perts, h=1e-5, xtol=1e-15,
               nthreads=0):
    """Central differences of the TI root: perts is a list of (lo, hi,
    kind), kind 0..4 = A, C, F, L, N of layer lo (= hi): dc/d(modulus);
    kind 5 = A and L of layers lo..hi scaled together: dc/dh."""
    a = _d7(thk, TA, TC, TF, TL, TN, rho)
    p = np.asarray(perts, np.int32).reshape(-1, 3)
    lo, hi, kind = (np.ascontiguousarray(p[:, i]) for i in range(3))
    out = np.zeros(len(p))
    r = lib().or_ti_root_fd(len(a[0]), *[_p(x, _f64p) for x in a], omega, c0, h, xtol * c0,
                            len(p), _p(lo, _i32p), _p(hi, _i32p), _p(kind, _i32p),
                            _p(out, _f64p), nthreads)
    if r != 0:
        raise RuntimeError(f"{r} TI roots failed")
    return out


def batch(node_off, depz, vs, per_off, periods, minthk, kernels=True, lsen=True, nthreads=0):
    """Oracle of the ragged batch (reference algorithms column by column,
    OpenMP over columns).  Outputs in the batch layout (see or_batch)."""
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    nz = np.diff(node_off)
    K = np.diff(per_off)
    sen_off = np.concatenate([[0], np.cumsum(K * nz)]).astype(np.int64)
    ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))]).astype(np.int64)
    pv = np.zeros(int(per_off[-1]))
    sen = [np.zeros(int(sen_off[-1])) for _ in range(3)] if kernels else [None] * 3
    ls = np.zeros(int(ls_off[-1]), np.float32) if lsen else None
    r = lib().or_batch(node_off.size - 1, _p(node_off, _i64p),
                       _p(np.ascontiguousarray(depz, np.float32), _f32p),
                       _p(np.ascontiguousarray(vs, np.float32), _f32p), _p(per_off, _i64p),
                       _p(np.ascontiguousarray(periods, np.float64), _f64p), ctypes.c_float(minthk),
                       _p(pv, _f64p), _p(sen_off, _i64p), _p(sen[0], _f64p), _p(sen[1], _f64p),
                       _p(sen[2], _f64p), _p(ls_off, _i64p), _p(ls, _f32p), nthreads)
    if r != 0:
        raise RuntimeError("oracle batch failed")
    return dict(pv=pv, sen_vs=sen[0], sen_vp=sen[1], sen_rho=sen[2], lsen=ls,
                sen_off=sen_off, ls_off=ls_off)


def batch_ti(node_off, depz, vs, per_off, periods, minthk, pv=None, root_tol=1e-6,
             nthreads=0):
    """Lsen_Gsc of a ragged batch (depthkernelTI's tregn96 + splice) at the
    given phase velocities pv (batch layout), or at surfdisp96's roots
    converged to root_tol.  Returns pv (the ones used), lsen and ls_off."""
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    nz = np.diff(node_off)
    K = np.diff(per_off)
    ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))]).astype(np.int64)
    ls = np.zeros(max(int(ls_off[-1]), 1), np.float32)
    pv_out = np.zeros(int(per_off[-1]))
    pv_in = None if pv is None else np.ascontiguousarray(pv, np.float64)
    r = lib().or_batch_ti(node_off.size - 1, _p(node_off, _i64p),
                          _p(np.ascontiguousarray(depz, np.float32), _f32p),
                          _p(np.ascontiguousarray(vs, np.float32), _f32p), _p(per_off, _i64p),
                          _p(np.ascontiguousarray(periods, np.float64), _f64p),
                          ctypes.c_float(minthk), _p(pv_in, _f64p), root_tol, _p(pv_out, _f64p),
                          _p(ls_off, _i64p), _p(ls, _f32p), nthreads)
    if r != 0:
        raise RuntimeError("oracle batch_ti failed")
    return dict(pv=pv_out, lsen=ls[:int(ls_off[-1])], ls_off=ls_off)


def batch_fd(node_off, depz, vs, per_off, periods, minthk, exact=False, tol=None, dln=None,
             nthreads=0):
    """Vs-type kernels of a ragged batch: the reference's arithmetic, or
    (exact=True) the exact-model checker (double model, unrounded roots, tol
    1e-13 and dln 1e-4 unless given).  Returns pv, sen_vs, sen_vp, sen_rho
    in the batch layout, sen_off and status."""
    node_off = np.ascontiguousarray(node_off, np.int64)
    per_off = np.ascontiguousarray(per_off, np.int64)
    nz = np.diff(node_off)
    K = np.diff(per_off)
    sen_off = np.concatenate([[0], np.cumsum(K * nz)]).astype(np.int64)
    pv = np.zeros(int(per_off[-1]))
    sen = [np.zeros(max(int(sen_off[-1]), 1)) for _ in range(3)]
    st = np.zeros(max(node_off.size - 1, 1), np.int32)
    tol = tol if tol is not None else (1e-13 if exact else 1e-6)
    dln = dln if dln is not None else (1e-4 if exact else 0.01)
    r = lib().or_batch_fd(node_off.size - 1, _p(node_off, _i64p),
                          _p(np.ascontiguousarray(depz, np.float32), _f32p),
                          _p(np.ascontiguousarray(vs, np.float32), _f32p), _p(per_off, _i64p),
                          _p(np.ascontiguousarray(periods, np.float64), _f64p),
                          ctypes.c_float(minthk), _p(pv, _f64p), _p(sen_off, _i64p),
                          _p(sen[0], _f64p), _p(sen[1], _f64p), _p(sen[2], _f64p),
                          2 if exact else 0, tol, ctypes.c_float(dln), _p(st, _i32p), nthreads)
    if r != 0:
        raise RuntimeError("oracle batch_fd failed")
    return dict(pv=pv, sen_vs=sen[0], sen_vp=sen[1], sen_rho=sen[2], sen_off=sen_off,
                status=st[:node_off.size - 1])


def grows(nvx, nvz, vels, sen_vs, sen_vp, sen_rho, lsen, ray_period, ray_id, cell_off, cell, fdm,
          fdmc=None, fdms=None, ftol=1e-4, cap=None):
    """Oracle of the G-row epilogue (CalSurfG_parallel.f90:2363-2400):
    sparse entries (rw float32, iw ray id, col 1-based parameter) and the
    entry count of every ray.  vels (nvx+2, nvz+2, nz) float32, kernels
    (nxy, K, nz) float64, lsen (nxy, K, nz-1) float32 or None."""
    vels = np.asfortranarray(vels, np.float32)
    nz = vels.shape[2]
    K = sen_vs.shape[1]
    f64 = lambda a: np.asfortranarray(a, np.float64)  # noqa: E731
    ls = None if lsen is None else np.asfortranarray(lsen, np.float32)
    cell_off = np.ascontiguousarray(cell_off, np.int64)
    nrays = cell_off.size - 1
    i32 = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
    f32 = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)  # noqa: E731
    if cap is None:
        cap = int(cell_off[-1]) * (nz - 1) * (3 if ls is not None else 1) + 1
    rw = np.zeros(cap, np.float32)
    iw = np.zeros(cap, np.int32)
    col = np.zeros(cap, np.int32)
    nnz = np.zeros(max(nrays, 1), np.int64)
    a = [i32(ray_period), i32(ray_id), i32(cell), f32(fdm), f32(fdmc), f32(fdms)]
    n = lib().or_grows(nvx, nvz, nz, K, _p(vels, _f32p), _p(f64(sen_vs), _f64p),
                       _p(f64(sen_vp), _f64p), _p(f64(sen_rho), _f64p), _p(ls, _f32p), nrays,
                       _p(a[0], _i32p), _p(a[1], _i32p), _p(cell_off, _i64p), _p(a[2], _i32p),
                       _p(a[3], _f32p), _p(a[4], _f32p), _p(a[5], _f32p), ctypes.c_float(ftol),
                       cap, _p(rw, _f32p), _p(iw, _i32p), _p(col, _i32p), _p(nnz, _i64p))
    if n < 0:
        raise RuntimeError("oracle grows: capacity exceeded or invalid cell")
    return rw[:n], iw[:n], col[:n], nnz[:nrays]


def azimap(lsen, gc, gs, ciso):
    """Oracle of FwdAzimuthalAniMap.f90:43-86.  lsen (nx*ny, K, nz-1) on the
    (nx, ny) grid, gc/gs (nx-2, ny-2, nz-1), ciso ((nx-2)*(ny-2), K).
    Returns cos, sin, amp, amp_rel, angle, each ((nx-2)*(ny-2), K) float32."""
    gc = np.asfortranarray(gc, np.float32)
    nvx, nvz, nzm1 = gc.shape
    nx, ny, nz = nvx + 2, nvz + 2, nzm1 + 1
    K = lsen.shape[1]
    out = [np.zeros((nvx * nvz, K), np.float32, order="F") for _ in range(5)]
    lib().or_azimap(nx, ny, nz, K, _p(np.asfortranarray(lsen, np.float32), _f32p), _p(gc, _f32p),
                    _p(np.asfortranarray(gs, np.float32), _f32p),
                    _p(np.asfortranarray(ciso, np.float64), _f64p), *[_p(o, _f32p) for o in out])
    return tuple(out)


def fmm_batch(params, pv, inst_period, scx, scz, rc_off, rcx, rcz, nthreads=0, fields=False):
    """Forward traveltimes of a data set (or_fmm_batch, fmm_oracle.c):
    pv (nx*ny, K) phase-velocity maps (x index fastest, float64), one
    instance per (period index, source) with its receivers in CSR rc_off;
    coordinates are colatitude and longitude in radians (float32), as
    Main_Jt.f90:412-431 converts them.  Returns the receiver times (float32)
    and, when fields, the coarse traveltime fields (ninst, nnx, nnz)."""
    P = params
    pv = np.asfortranarray(pv, np.float64)
    ninst = len(inst_period)
    rc_off = np.ascontiguousarray(rc_off, np.int64)
    times = np.zeros(max(int(rc_off[-1]), 1), np.float32)
    nnx, nnz = (P.nx - 3) * P.gdx + 1, (P.ny - 3) * P.gdz + 1
    ttn = np.zeros((ninst, nnx, nnz), np.float32) if fields else None
    nthreads = nthreads or (os.cpu_count() or 1)
    r = lib().or_fmm_batch(ctypes.byref(P), _p(pv, _f64p), ninst,
                           _p(np.ascontiguousarray(inst_period, np.int32), _i32p),
                           _p(np.ascontiguousarray(scx, np.float32), _f32p),
                           _p(np.ascontiguousarray(scz, np.float32), _f32p), _p(rc_off, _i64p),
                           _p(np.ascontiguousarray(rcx, np.float32), _f32p),
                           _p(np.ascontiguousarray(rcz, np.float32), _f32p), _p(times, _f32p),
                           None if ttn is None else _p(ttn, _f32p), nthreads)
    if r:
        raise RuntimeError(f"oracle fmm_batch: error {r}")
    return (times[:int(rc_off[-1])], ttn) if fields else times[:int(rc_off[-1])]


def fmm_travel(veln, gox, goz, dnx, dnz, scx, scz, earth=6371.0, fom=1, snb=0.5):
    """One traveltime field on a given grid (travel with urg = 0): veln
    (nnx, nnz) float32 (x outer); returns ttn (nnx, nnz) and the status."""
    veln = np.ascontiguousarray(veln, np.float32)
    nnx, nnz = veln.shape
    ttn = np.zeros_like(veln)
    st = np.zeros(veln.shape, np.int32)
    r = lib().or_fmm_travel(nnx, nnz, gox, goz, dnx, dnz, earth, fom, snb, _p(veln, _f32p), scx,
                            scz, _p(ttn, _f32p), _p(st, _i32p))
    if r:
        raise RuntimeError(f"oracle fmm_travel: error {r}")
    return ttn, st
