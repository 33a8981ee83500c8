"""Loader of the in-tree CUDA library libdazi_dk.so (C-ABI, include/dazi_dk.h).

The library must be built (python -m dazi_current_release_b200.build); there is
no CPU fallback: a missing library or a machine without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)
_int = ctypes.c_int

DAZI_OK = 0
DAZI_WARN_NOROOT = 1
DAZI_ERR_BADARG = -1
DAZI_ERR_LIMITS = -2
DAZI_ERR_CUDA = -3
DAZI_ERR_TIMEOUT = -4
DAZI_ERR_NOMEM = -5
DAZI_ERR_NODEVICE = -6
DAZI_ERR_MODEL = -7
FORM_PLAIN = 0
FORM_ADJOINT = 1
FORM_SCAN_FP32 = 2      # flag: FP32 coarse scan verified in FP64 (default: all FP64)
FORM_LOVE = 4           # flag: Love waves (surfdisp96 iwave = 1), plain or adjoint form
FORM_GROUP = 8          # flag: group velocity (igr > 0), plain or adjoint form
FORM_FAST_ROOT = 16     # flag: Brent refinement of the reference's bracket (Rayleigh phase)
FORM_FULL_STACK = 32    # flag: adjoint and Lsen_Gsc sweeps over the whole stack (no depth cut)

# every symbol include/dazi_dk.h declares
EXPORTS = (
    "dazi_dk_iso", "dazi_dk_iso_vpvsrho", "dazi_dk_last_status", "dazi_dk_iso_dev",
    "dazi_dk_last_error", "dazi_dk_version", "dazi_dk_finalize", "dazi_dk_fp64_peak", "dazi_dk_last_work",
    "dazi_dk_ti", "dazi_dk_fused", "dazi_dk_fused_dev", "dazi_dk_last_launches",
    "dazi_dk_iso_noalloc_dev", "dazi_dk_batch", "dazi_dk_batch_dev", "dazi_dk_set_timing",
    "dazi_dk_last_timing", "dazi_dk_last_items", "dazi_dk_plan_create", "dazi_dk_plan_launch",
    "dazi_dk_plan_status", "dazi_dk_plan_config", "dazi_dk_plan_destroy", "dazi_dk_grows_dev",
    "dazi_dk_azimuthal_map_dev", "dazi_lsmr", "dazi_lsmr_dev", "dazi_fmm_default_params",
    "dazi_fmm_batch", "dazi_fmm_batch_dev", "dazi_fmm_times",
)


class FmmParams(ctypes.Structure):
    """dazi_fmm_params (include/dazi_dk.h): model grid and traveltime-solver
    settings."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("goxd", ctypes.c_float),
                ("gozd", ctypes.c_float), ("dvxd", ctypes.c_float), ("dvzd", ctypes.c_float),
                ("gdx", ctypes.c_int), ("gdz", ctypes.c_int), ("asgr", ctypes.c_int),
                ("sgdl", ctypes.c_int), ("sgs", ctypes.c_int), ("fom", ctypes.c_int),
                ("snb", ctypes.c_float), ("earth", ctypes.c_float)]


class DaziError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dazi_dk error {code}: {msg}")
        self.code = code


_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libdazi_dk.so and declare the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise FileNotFoundError(f"{path} is not built")
        _build.build()
    L = ctypes.CDLL(path)
    ip = ctypes.POINTER(ctypes.c_int)
    fp = _f32p
    L.dazi_dk_iso.argtypes = [ip, ip, ip, fp, _f64p, _f64p, _f64p, _f64p, ip, ip, ip, _f64p, fp,
                              fp, _int, _int, _int]
    L.dazi_dk_iso.restype = _int
    L.dazi_dk_iso_vpvsrho.argtypes = [ip, ip, ip, fp, fp, fp, _f64p, _f64p, _f64p, _f64p, ip, ip,
                                      ip, _f64p, fp, fp, _int, _int, _int]
    L.dazi_dk_iso_vpvsrho.restype = _int
    L.dazi_dk_last_status.argtypes = [_i32p, ctypes.c_longlong]
    L.dazi_dk_last_status.restype = _int
    vp_ = ctypes.c_void_p
    L.dazi_dk_iso_dev.argtypes = [_int, _int, _int, vp_, vp_, vp_, vp_, vp_, vp_, vp_, _int, vp_,
                                  vp_, ctypes.c_float, _int, _int, _int, vp_, vp_]
    L.dazi_dk_iso_dev.restype = _int
    L.dazi_dk_ti.argtypes = [ip, ip, ip, fp, _f64p, ip, ip, ip, _f64p, fp, fp, fp, _int, _int]
    L.dazi_dk_ti.restype = _int
    L.dazi_dk_fused.argtypes = [ip, ip, ip, fp, fp, fp, _f64p, _f64p, _f64p, _f64p, fp, ip, ip, ip,
                                _f64p, fp, fp, _int, _int, _int]
    L.dazi_dk_fused.restype = _int
    L.dazi_dk_fused_dev.argtypes = [_int, _int, _int, vp_, vp_, vp_, vp_, vp_, vp_, vp_, vp_, _int,
                                    vp_, vp_, ctypes.c_float, _int, _int, _int, vp_, vp_]
    L.dazi_dk_fused_dev.restype = _int
    # dazi_dk_iso_dev's list without `form` (the entry runs the plain form only)
    L.dazi_dk_iso_noalloc_dev.argtypes = [_int, _int, _int, vp_, vp_, vp_, vp_, vp_, vp_, vp_, _int,
                                          vp_, vp_, ctypes.c_float, _int, _int, vp_, vp_]
    L.dazi_dk_iso_noalloc_dev.restype = _int
    i64p = ctypes.POINTER(ctypes.c_longlong)
    ll = ctypes.c_longlong
    L.dazi_dk_batch.argtypes = [ll, i64p, fp, fp, fp, fp, i64p, _f64p, ctypes.c_float, _f64p, i64p,
                                _f64p, _f64p, _f64p, i64p, fp, _int, _i32p]
    L.dazi_dk_batch.restype = _int
    L.dazi_dk_batch_dev.argtypes = [ll] + [vp_] * 7 + [ctypes.c_float] + [vp_] * 7 + [_int, vp_, vp_]
    L.dazi_dk_batch_dev.restype = _int
    L.dazi_dk_set_timing.argtypes = [_int]
    L.dazi_dk_set_timing.restype = _int
    L.dazi_dk_last_timing.argtypes = [ctypes.POINTER(ctypes.c_char_p), _f64p, _int]
    L.dazi_dk_last_timing.restype = _int
    L.dazi_dk_last_launches.argtypes = []
    L.dazi_dk_last_launches.restype = _int
    L.dazi_dk_last_error.argtypes = []
    L.dazi_dk_last_error.restype = ctypes.c_char_p
    L.dazi_dk_version.argtypes = []
    L.dazi_dk_version.restype = _int
    L.dazi_dk_last_work.argtypes = [ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.dazi_dk_last_work.restype = _int
    L.dazi_dk_last_items.argtypes = [ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.dazi_dk_last_items.restype = _int
    L.dazi_dk_plan_create.argtypes = ([ll] + [vp_] * 7 + [ctypes.c_float] + [vp_] * 7 +
                                      [_int, vp_, _int, vp_, ctypes.POINTER(ctypes.c_void_p)])
    L.dazi_dk_plan_create.restype = _int
    L.dazi_dk_plan_launch.argtypes = [vp_, vp_]
    L.dazi_dk_plan_launch.restype = _int
    L.dazi_dk_plan_status.argtypes = [vp_]
    L.dazi_dk_plan_status.restype = _int
    L.dazi_dk_plan_config.argtypes = [vp_, _i32p, _i32p, _i32p, ctypes.POINTER(ctypes.c_float)]
    L.dazi_dk_plan_config.restype = _int
    L.dazi_dk_plan_destroy.argtypes = [vp_]
    L.dazi_dk_plan_destroy.restype = _int
    L.dazi_dk_grows_dev.argtypes = ([_int] * 4 + [vp_] * 5 + [ll] + [vp_] * 7 + [ctypes.c_float, ll] +
                                    [vp_] * 4 + [ctypes.POINTER(ctypes.c_longlong), vp_])
    L.dazi_dk_grows_dev.restype = _int
    L.dazi_dk_azimuthal_map_dev.argtypes = [_int] * 4 + [vp_] * 10
    L.dazi_dk_azimuthal_map_dev.restype = _int
    ll_p = ctypes.POINTER(ctypes.c_longlong)
    L.dazi_lsmr.argtypes = [ip, ip, ll_p, ll_p, ip, fp, _f64p, _f64p, _f64p, _f64p, _f64p, ip, ip,
                            ip, _f64p, ip, ip, _f64p, _f64p, _f64p, _f64p, _f64p]
    L.dazi_lsmr.restype = _int
    L.dazi_lsmr_dev.argtypes = [_int, _int, ll, vp_, vp_, vp_, _int, vp_, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, _int, vp_,
                                ip, ip, _f64p, vp_]
    L.dazi_lsmr_dev.restype = _int
    L.dazi_dk_fp64_peak.argtypes = [_f64p]
    L.dazi_dk_fp64_peak.restype = _int
    L.dazi_dk_finalize.argtypes = []
    L.dazi_dk_finalize.restype = None
    fpp = ctypes.POINTER(FmmParams)
    L.dazi_fmm_default_params.argtypes = [fpp, _int, _int] + [ctypes.c_float] * 4
    L.dazi_fmm_default_params.restype = None
    L.dazi_fmm_batch.argtypes = [fpp, _f64p, _int, _int, ip, fp, fp, ll_p, fp, fp, fp, fp]
    L.dazi_fmm_batch.restype = _int
    L.dazi_fmm_batch_dev.argtypes = [fpp, vp_, _int, _int] + [vp_] * 8 + [vp_]
    L.dazi_fmm_batch_dev.restype = _int
    L.dazi_fmm_times.argtypes = [ip] * 6 + [_f64p, ip, ip, ip, fp, fp, fp, fp, fp, fp, fp, fp, ll_p, fp]
    L.dazi_fmm_times.restype = _int
    _lib = L
    return L


def check(code: int) -> int:
    """Raise DaziError for negative return codes; pass 0/1 through."""
    if code < 0:
        msg = load().dazi_dk_last_error().decode(errors="replace")
        raise DaziError(code, msg)
    return code


def last_timing(cap: int = 16) -> dict:
    """Per-phase milliseconds of the last call (needs dazi_dk_set_timing(1))."""
    L = load()
    names = (ctypes.c_char_p * cap)()
    ms = (ctypes.c_double * cap)()
    n = check(L.dazi_dk_last_timing(names, ms, cap))
    return {names[i].decode(): ms[i] for i in range(n)}
