"""C-ABI checks that need no GPU: the library loads, exports every symbol the
public header declares, and rejects bad arguments before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from dazi_current_release_b200 import _lib, depthkernel as dkmod
from dazi_current_release_b200.depthkernel import DepthKernelError, depthkernelTI, resolve_form

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "dazi_dk.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dazi_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = header_functions()
    assert len(names) >= 7
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTS)


def header_arity():
    """Parameter count of every function the public header declares."""
    text = open(os.path.join(ROOT, "include", "dazi_dk.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(dazi_\w+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = params.strip()
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_bindings_match_header_arity():
    """Each ctypes binding declares as many arguments as the C prototype
    (a mismatch shifts arguments silently, e.g. an int into a pointer)."""
    L = _lib.load()
    arity = header_arity()
    assert set(arity) == set(_lib.EXPORTS)
    for name, n in arity.items():
        assert len(getattr(L, name).argtypes) == n, name


def test_version():
    assert _lib.load().dazi_dk_version() >= 100


def _call_iso(nx=2, ny=2, nz=3, iwave=2, igr=0, K=2, depz=(0.0, 3.0, 6.0), vel=3.5,
              col_start=1, col_count=None, form=0, periods=(5.0, 10.0)):
    L = _lib.load()
    vel = np.full((nx, ny, nz), vel, np.float32, order="F")
    pv = np.zeros((nx * ny, K), order="F")
    t = np.asarray(periods, np.float64)
    d = np.asarray(depz, np.float32)
    ci = ctypes.c_int
    f64p = ctypes.POINTER(ctypes.c_double)
    f32p = ctypes.POINTER(ctypes.c_float)
    if col_count is None:
        col_count = nx * ny
    return L.dazi_dk_iso(ctypes.byref(ci(nx)), ctypes.byref(ci(ny)), ctypes.byref(ci(nz)),
                         vel.ctypes.data_as(f32p), pv.ctypes.data_as(f64p), None, None, None,
                         ctypes.byref(ci(iwave)), ctypes.byref(ci(igr)), ctypes.byref(ci(K)),
                         t.ctypes.data_as(f64p), d.ctypes.data_as(f32p),
                         ctypes.byref(ctypes.c_float(4.0)), col_start, col_count, form)


@pytest.mark.parametrize("kw,code", [
    (dict(iwave=3), _lib.DAZI_ERR_BADARG),              # neither Love nor Rayleigh
    (dict(iwave=0), _lib.DAZI_ERR_BADARG),
    (dict(igr=1, form=_lib.FORM_SCAN_FP32), _lib.DAZI_ERR_BADARG),   # FP32 scan: Rayleigh phase
    (dict(iwave=1, form=_lib.FORM_ADJOINT | _lib.FORM_SCAN_FP32), _lib.DAZI_ERR_BADARG),
    (dict(form=_lib.FORM_LOVE), _lib.DAZI_ERR_BADARG),  # wave type goes through iwave here
    (dict(form=_lib.FORM_GROUP), _lib.DAZI_ERR_BADARG),
    (dict(depz=(0.0, 3.0, 3.0)), _lib.DAZI_ERR_BADARG),  # not increasing
    (dict(col_start=0), _lib.DAZI_ERR_BADARG),
    (dict(col_start=3, col_count=3), _lib.DAZI_ERR_BADARG),
    (dict(vel=-1.0), _lib.DAZI_ERR_BADARG),
    (dict(vel=float("nan")), _lib.DAZI_ERR_BADARG),
    (dict(periods=(5.0, 0.0)), _lib.DAZI_ERR_BADARG),
    (dict(nz=1, depz=(0.0,)), _lib.DAZI_ERR_LIMITS),
    (dict(form=7), _lib.DAZI_ERR_BADARG),
    (dict(form=64), _lib.DAZI_ERR_BADARG),              # unknown flag
    (dict(iwave=1, form=_lib.FORM_ADJOINT | _lib.FORM_FAST_ROOT), _lib.DAZI_ERR_BADARG),
    (dict(igr=1, form=_lib.FORM_ADJOINT | _lib.FORM_FAST_ROOT), _lib.DAZI_ERR_BADARG),
])
def test_bad_arguments_rejected_without_device(kw, code):
    assert _call_iso(**kw) == code
    assert len(_lib.load().dazi_dk_last_error()) > 0


@pytest.mark.parametrize("iwave,igr,form", [(1, 0, 0), (2, 1, 0), (1, 1, 0), (2, 5, 0), (1, 0, 1),
                                            (2, 1, 1), (1, 1, 1), (2, 0, 17), (2, 0, 19)])
def test_love_and_group_pass_validation(iwave, igr, form):
    """Love (iwave = 1) and group velocity (igr > 0) are accepted by the
    plain and the adjoint form; without a GPU the call then stops at the
    device check."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    assert _call_iso(iwave=iwave, igr=igr, form=form) == _lib.DAZI_ERR_NODEVICE


@pytest.mark.parametrize("iwave,igr", [(1, 0), (2, 1)])
def test_gc_gs_kernel_is_rayleigh_phase_only(iwave, igr):
    with pytest.raises(_lib.DaziError) as ei:
        depthkernelTI(2, 2, 3, np.full((2, 2, 3), 3.5, np.float32, order="F"), iwave, igr,
                      2, np.array([5.0, 10.0]), np.array([0.0, 3.0, 6.0], np.float32), 4.0)
    assert ei.value.code == _lib.DAZI_ERR_BADARG
    assert "Rayleigh" in _lib.load().dazi_dk_last_error().decode()


def test_no_device_is_a_loud_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(_lib.DaziError) as ei:
        _lib.check(_call_iso())
    assert ei.value.code == _lib.DAZI_ERR_NODEVICE


def test_backend_dispatch(monkeypatch):
    monkeypatch.setenv("DAZI_DEPTHKERNEL_BACKEND", "b200")
    assert resolve_form() == _lib.FORM_PLAIN
    monkeypatch.setenv("DAZI_DEPTHKERNEL_BACKEND", "b200_adjoint")
    assert resolve_form() == _lib.FORM_ADJOINT
    monkeypatch.setenv("DAZI_DEPTHKERNEL_BACKEND", "default_fortran_fd")
    with pytest.raises(DepthKernelError) as ei:
        resolve_form()
    assert ei.value.code == 9201
    monkeypatch.delenv("DAZI_DEPTHKERNEL_BACKEND")
    assert resolve_form() == _lib.FORM_PLAIN
