"""Host-side mirror of the reference depth-kernel drivers.

`depthkernel` follows code/src_inv_iso_joint/CalSurfG.f90:1-113: same
arguments and meaning (vel(nx,ny,nz) real*4, tRc(kmaxRc) real*8, depz(nz),
minthk = sublayer count, iwave = 2, igr = 0), same Fortran-order outputs
pvRc(nx*ny,kmaxRc) and sen_*Rc(nx*ny,kmaxRc,nz).  The backend is chosen by
the environment variable DAZI_DEPTHKERNEL_BACKEND as in CalSurfG.f90:37-58;
this library provides

    b200          perturb-and-recompute form (the reference's kernels)
    b200_adjoint  implicit differentiation of the root (adjoint form)

An unknown name raises DepthKernelError(9201), the code the reference uses
for an unknown backend (depthkernelTI.f90:83).  Every call runs on the GPU;
there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

BACKENDS = {"b200": _lib.FORM_PLAIN, "b200_adjoint": _lib.FORM_ADJOINT,
            "b200_adjoint_fp32scan": _lib.FORM_ADJOINT | _lib.FORM_SCAN_FP32}
ENV_ISO = "DAZI_DEPTHKERNEL_BACKEND"
ENV_TI = "DAZI_DEPTHKERNEL_TI_BACKEND"


class DepthKernelError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"depth kernel stop {code}: {msg}")
        self.code = code


def resolve_form(env: str = ENV_ISO, default: str = "b200") -> int:
    name = os.environ.get(env, "").strip() or default
    if name not in BACKENDS:
        raise DepthKernelError(9201, f"unknown depth kernel backend {name!r} "
                                     f"(this library provides {sorted(BACKENDS)})")
    return BACKENDS[name]


def _f32(a, shape=None, order="F"):
    a = np.asarray(a, dtype=np.float32, order=order)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape, order=order)
    return a


def _ptr(a, ct):
    return None if a is None else a.ctypes.data_as(ct)


def _run_iso(nx, ny, nz, vel, vp, rho, iwave, igr, kmaxRc, tRc, depz, minthk, form,
             col_start, col_count, kernels, pvRc=None, sen=None):
    L = _lib.load()
    vel = _f32(vel, (nx, ny, nz))
    if vp is not None:
        vp = _f32(vp, (nx, ny, nz))
        rho = _f32(rho, (nx, ny, nz))
    tRc = np.ascontiguousarray(tRc, dtype=np.float64)
    depz = np.ascontiguousarray(depz, dtype=np.float32)
    if tRc.size != kmaxRc or depz.size != nz:
        raise ValueError("tRc must have kmaxRc entries and depz nz entries")
    nxy = nx * ny
    if col_count is None:
        col_count = nxy - col_start + 1
    if pvRc is None:
        pvRc = np.zeros((nxy, kmaxRc), np.float64, order="F")
    if kernels and sen is None:
        sen = tuple(np.zeros((nxy, kmaxRc, nz), np.float64, order="F") for _ in range(3))
    f64p = ctypes.POINTER(ctypes.c_double)
    f32p = ctypes.POINTER(ctypes.c_float)
    ci = ctypes.c_int
    args_head = (ctypes.byref(ci(nx)), ctypes.byref(ci(ny)), ctypes.byref(ci(nz)), _ptr(vel, f32p))
    args_out = (_ptr(pvRc, f64p),) + (tuple(_ptr(s, f64p) for s in sen) if kernels else (None,) * 3)
    args_tail = (ctypes.byref(ci(iwave)), ctypes.byref(ci(igr)), ctypes.byref(ci(kmaxRc)),
                 _ptr(tRc, f64p), _ptr(depz, f32p), ctypes.byref(ctypes.c_float(minthk)),
                 int(col_start), int(col_count), int(form))
    if vp is None:
        rc = L.dazi_dk_iso(*args_head, *args_out, *args_tail)
    else:
        rc = L.dazi_dk_iso_vpvsrho(*args_head, _ptr(vp, f32p), _ptr(rho, f32p), *args_out,
                                   *args_tail)
    _lib.check(rc)
    if kernels:
        return (pvRc,) + tuple(sen)
    return (pvRc,)


def depthkernel(nx, ny, nz, vel, iwave, igr, kmaxRc, tRc, depz, minthk, *, form=None,
                col_start=1, col_count=None, kernels=True):
    """depthkernel(nx,ny,nz,vel,pvRc,sen_vsRc,sen_vpRc,sen_rhoRc,iwave,igr,kmaxRc,tRc,depz,minthk)

    Returns (pvRc, sen_vsRc, sen_vpRc, sen_rhoRc) as Fortran-ordered arrays
    (pvRc only when kernels=False).  form: FORM_PLAIN / FORM_ADJOINT, or
    None to read DAZI_DEPTHKERNEL_BACKEND.  iwave 2 (Rayleigh) or 1 (Love),
    igr 0 (phase) or > 0 (group velocity), as surfdisp96 takes them, in
    either form.
    """
    if form is None:
        form = resolve_form(ENV_ISO)
    return _run_iso(nx, ny, nz, vel, None, None, iwave, igr, kmaxRc, tRc, depz, minthk, form,
                    col_start, col_count, kernels)


def depthkernel_vpvsrho(nx, ny, nz, vel, vp, rho, iwave, igr, kmaxRc, tRc, depz, minthk, *,
                        form=None, col_start=1, col_count=None, kernels=True):
    """depthkernel with explicit Vp and rho node arrays (nx,ny,nz)."""
    if form is None:
        form = resolve_form(ENV_ISO)
    return _run_iso(nx, ny, nz, vel, vp, rho, iwave, igr, kmaxRc, tRc, depz, minthk, form,
                    col_start, col_count, kernels)


def _run_fused(nx, ny, nz, vel, vp, rho, iwave, igr, kmaxRc, tRc, depz, minthk, form,
               col_start, col_count, kernels, lsen, pvRc=None, sen=None, Lsen=None):
    L = _lib.load()
    vel = _f32(vel, (nx, ny, nz))
    if vp is not None:
        vp = _f32(vp, (nx, ny, nz))
        rho = _f32(rho, (nx, ny, nz))
    tRc = np.ascontiguousarray(tRc, dtype=np.float64)
    depz = np.ascontiguousarray(depz, dtype=np.float32)
    if tRc.size != kmaxRc or depz.size != nz:
        raise ValueError("tRc must have kmaxRc entries and depz nz entries")
    nxy = nx * ny
    if col_count is None:
        col_count = nxy - col_start + 1
    if pvRc is None:
        pvRc = np.zeros((nxy, kmaxRc), np.float64, order="F")
    if kernels and sen is None:
        sen = tuple(np.zeros((nxy, kmaxRc, nz), np.float64, order="F") for _ in range(3))
    if lsen and Lsen is None:
        Lsen = np.zeros((nxy, kmaxRc, nz - 1), np.float32, order="F")
    f64p = ctypes.POINTER(ctypes.c_double)
    f32p = ctypes.POINTER(ctypes.c_float)
    ci = ctypes.c_int
    rc = L.dazi_dk_fused(ctypes.byref(ci(nx)), ctypes.byref(ci(ny)), ctypes.byref(ci(nz)),
                         _ptr(vel, f32p), _ptr(vp, f32p), _ptr(rho, f32p), _ptr(pvRc, f64p),
                         *(tuple(_ptr(x, f64p) for x in sen) if kernels else (None,) * 3),
                         _ptr(Lsen, f32p) if lsen else None,
                         ctypes.byref(ci(iwave)), ctypes.byref(ci(igr)), ctypes.byref(ci(kmaxRc)),
                         _ptr(tRc, f64p), _ptr(depz, f32p), ctypes.byref(ctypes.c_float(minthk)),
                         int(col_start), int(col_count), int(form))
    _lib.check(rc)
    out = (pvRc,)
    if kernels:
        out += tuple(sen)
    if lsen:
        out += (Lsen,)
    return out


def depthkernelTI(nx, ny, nz, vel, iwave, igr, kmaxRc, tRc, depz, minthk, *, vp=None, rho=None,
                  col_start=1, col_count=None):
    """depthkernelTI(nx,ny,nz,vel,pvRc,iwave,igr,kmaxRc,tRc,depz,minthk,Lsen_Gsc)

    code/src_inv_iso_joint/depthkernelTI.f90:2-193.  Returns
    (pvRc, Lsen_Gsc): pvRc(nx*ny,kmaxRc) real*8 and Lsen_Gsc(nx*ny,kmaxRc,nz-1)
    real*4, Fortran order.  DAZI_DEPTHKERNEL_TI_BACKEND must be unset or b200.
    """
    name = os.environ.get(ENV_TI, "").strip() or "b200"
    if name not in ("b200", "b200_adjoint"):
        raise DepthKernelError(9201, f"unknown Depth kernel TI backend {name!r}")
    return _run_fused(nx, ny, nz, vel, vp, rho, iwave, igr, kmaxRc, tRc, depz, minthk,
                      _lib.FORM_PLAIN, col_start, col_count, False, True)


def depthkernel_fused(nx, ny, nz, vel, iwave, igr, kmaxRc, tRc, depz, minthk, *, vp=None,
                      rho=None, form=None, col_start=1, col_count=None):
    """Both stages with one phase-velocity pass: returns
    (pvRc, sen_vsRc, sen_vpRc, sen_rhoRc, Lsen_Gsc)."""
    if form is None:
        form = resolve_form(ENV_ISO)
    return _run_fused(nx, ny, nz, vel, vp, rho, iwave, igr, kmaxRc, tRc, depz, minthk, form,
                      col_start, col_count, True, True)


def last_status(nxy: int) -> np.ndarray:
    st = np.zeros(nxy, np.int32)
    _lib.check(_lib.load().dazi_dk_last_status(st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                               nxy))
    return st
