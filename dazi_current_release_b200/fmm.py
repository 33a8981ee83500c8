"""First-arrival traveltimes of a surface-wave data set on the GPU.

The reference computes, for every (period, source), the traveltime field
through the period's phase-velocity map by fast marching on the refined
spherical grid and interpolates it at the receivers
(code/src_inv_iso_joint/CalSurfG_parallel.f90:2061-2340).  These functions
run that computation for all instances at once through the library's C-ABI
(dazi_fmm_batch / dazi_fmm_batch_dev), with the reference's arithmetic:
the times and fields are the reference's values.

Coordinates are colatitude and longitude in radians (float32), as
Main_Jt.f90:412-431 converts a data file's latitudes and longitudes
(``colatitude`` and ``longitude`` below do the same).  ``pv`` holds the
phase-velocity maps, one column of nx*ny values per period (the latitude
index fastest), as the depth-kernel stage writes pvRc.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_PI = np.float32(3.1415926535898)


def colatitude(lat):
    """(90 - lat) * pi / 180 in real*4, as the reference converts it."""
    return (np.float32(90.0) - np.asarray(lat, np.float32)) * _PI / np.float32(180.0)


def longitude(lon):
    return np.asarray(lon, np.float32) * _PI / np.float32(180.0)


def params(nx, ny, goxd, gozd, dvxd, dvzd, **settings) -> _lib.FmmParams:
    """The reference's solver settings for an nx x ny model grid whose first
    inner vertex is (goxd, gozd) degrees with spacing (dvxd, dvzd); keyword
    arguments override gdx, gdz, asgr, sgdl, sgs, fom, snb, earth."""
    p = _lib.FmmParams()
    _lib.load().dazi_fmm_default_params(ctypes.byref(p), nx, ny, goxd, gozd, dvxd, dvzd)
    for k, v in settings.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown setting {k}")
        setattr(p, k, v)
    return p


def field_shape(p) -> tuple:
    """(nnx, nnz) of the propagation grid."""
    return (p.nx - 3) * p.gdx + 1, (p.ny - 3) * p.gdz + 1


def travel_times(p, pv, inst_period, scx, scz, rc_off, rcx, rcz, fields=False):
    """Receiver times (float32, in the order of the receivers) of every
    instance s: period column inst_period[s] (0-based), source (scx[s],
    scz[s]), receivers rc_off[s] .. rc_off[s+1]-1.  With fields, also the
    coarse traveltime fields, (ninst, nnx, nnz) float32.  Host arrays."""
    L = _lib.load()
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    pv = np.asfortranarray(pv, np.float64)
    if pv.ndim != 2 or pv.shape[0] != p.nx * p.ny:
        raise ValueError("pv must be (nx*ny, nper)")
    inst_period = np.ascontiguousarray(inst_period, np.int32)
    rc_off = np.ascontiguousarray(rc_off, np.int64)
    ninst = inst_period.size
    if rc_off.size != ninst + 1:
        raise ValueError("rc_off must have ninst + 1 entries")
    nrc = int(rc_off[-1])
    times = np.zeros(max(nrc, 1), np.float32)
    ttn = np.zeros((ninst, *field_shape(p)), np.float32) if fields else None
    f32 = ctypes.c_float
    _lib.check(L.dazi_fmm_batch(ctypes.byref(p), P(pv, ctypes.c_double), pv.shape[1], ninst,
                                P(inst_period, ctypes.c_int),
                                P(np.ascontiguousarray(scx, np.float32), f32),
                                P(np.ascontiguousarray(scz, np.float32), f32),
                                P(rc_off, ctypes.c_longlong),
                                P(np.ascontiguousarray(rcx, np.float32), f32),
                                P(np.ascontiguousarray(rcz, np.float32), f32), P(times, f32),
                                None if ttn is None else P(ttn, f32)))
    return (times[:nrc], ttn) if fields else times[:nrc]


def travel_times_dev(p, pv, inst_period, scx, scz, rc_off, rcx, rcz, fields=False, stream=None):
    """travel_times on torch CUDA tensors (pv float64 (nper, nx*ny) rows or a
    flat column-major (nx*ny, nper) buffer, inst_period int32, coordinates
    float32, rc_off int64), stream-ordered on `stream` (default: torch's
    current stream).  Returns CUDA tensors."""
    import torch
    L = _lib.load()
    dev = pv.device
    for name, t, dt in (("pv", pv, torch.float64), ("inst_period", inst_period, torch.int32),
                        ("scx", scx, torch.float32), ("scz", scz, torch.float32),
                        ("rc_off", rc_off, torch.int64), ("rcx", rcx, torch.float32),
                        ("rcz", rcz, torch.float32)):
        if t.device != dev or t.dtype != dt or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous {dt} tensor on {dev}")
    nper = pv.numel() // (p.nx * p.ny)
    ninst = inst_period.numel()
    nrc = int(rc_off[-1].item())
    times = torch.zeros(max(nrc, 1), dtype=torch.float32, device=dev)
    ttn = torch.zeros((ninst, *field_shape(p)), dtype=torch.float32, device=dev) if fields else None
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    V = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _lib.check(L.dazi_fmm_batch_dev(ctypes.byref(p), V(pv), nper, ninst, V(inst_period), V(scx),
                                    V(scz), V(rc_off), V(rcx), V(rcz), V(times),
                                    None if ttn is None else V(ttn), ctypes.c_void_p(st.cuda_stream)))
    return (times[:nrc], ttn) if fields else times[:nrc]
