"""The reference's output formats for the stage's results (host side).

    write_period_phasev   WTPeriodPhaseV, Main_Jt.f90:2019-2038: one line per
                          (period, jj, ii) of the inner grid, '(5f10.4)':
                          latitude, longitude, period, phase velocity
    write_azimuthal_map   FwdAzimuthalAniMap.f90:67-84, '(10f10.5)': position,
                          period, c_iso, fast-axis angle, relative and absolute
                          amplitude, the cos and sin sums
    dump_depthkernel /    depthkernel_dump_arrays (CalSurfG.f90:117-140),
    dump_depthkernel_ti   depthkernelTI_dump_arrays (depthkernelTI.f90:195-213):
                          unformatted stream files of the Fortran-order arrays
    read_dump             the inverse of the dumps

Grid positions are real*4 in the reference (gozd + (jj-1) dvzd, goxd -
(ii-1) dvxd) and are formed in float32 here.
"""
from __future__ import annotations

import os

import numpy as np


def fortran_f(x, w, d):
    """Fortran Fw.d of one value ('*' * w when it does not fit)."""
    s = f"{float(x):{w}.{d}f}"
    return "*" * w if len(s) > w else s


def _pos(goxd, gozd, dvxd, dvzd, ii, jj):
    f = np.float32
    lat = f(f(gozd) + f(jj - 1) * f(dvzd))
    lon = f(f(goxd) - f(ii - 1) * f(dvxd))
    return lat, lon


def write_period_phasev(path, nx, ny, gozd, goxd, dvzd, dvxd, tRc, pv_inner):
    """pv_inner ((nx-2)*(ny-2), K): the inner columns, (jj-1)*(nx-2) + ii-1."""
    pv_inner = np.asarray(pv_inner, np.float64)
    with open(path, "w") as f:
        for tt, T in enumerate(np.asarray(tRc, np.float64)):
            for jj in range(1, ny - 1):
                for ii in range(1, nx - 1):
                    lat, lon = _pos(goxd, gozd, dvxd, dvzd, ii, jj)
                    v = pv_inner[(jj - 1) * (nx - 2) + ii - 1, tt]
                    f.write("".join(fortran_f(x, 10, 4) for x in (lat, lon, T, v)) + "\n")


def write_azimuthal_map(path, nx, ny, gozd, goxd, dvzd, dvxd, tRc, ciso, angle, amp_rel, amp,
                        cos_sum, sin_sum):
    """All per-(inner column, period) arrays ((nx-2)*(ny-2), K)."""
    with open(path, "w") as f:
        for tt, T in enumerate(np.asarray(tRc, np.float64)):
            for jj in range(1, ny - 1):
                for ii in range(1, nx - 1):
                    lat, lon = _pos(goxd, gozd, dvxd, dvzd, ii, jj)
                    o = (jj - 1) * (nx - 2) + ii - 1
                    vals = (lat, lon, T, np.float32(ciso[o, tt]), angle[o, tt], amp_rel[o, tt],
                            amp[o, tt], cos_sum[o, tt], sin_sum[o, tt])
                    f.write("".join(fortran_f(x, 10, 5) for x in vals) + "\n")


def _stream(path, a, dtype):
    np.asarray(a, dtype).ravel(order="F").tofile(path)


def dump_depthkernel(dump_dir, pvRc, sen_vsRc, sen_vpRc, sen_rhoRc):
    os.makedirs(dump_dir, exist_ok=True)
    _stream(os.path.join(dump_dir, "pv_depthkernel.bin"), pvRc, np.float64)
    _stream(os.path.join(dump_dir, "sen_vs_depthkernel.bin"), sen_vsRc, np.float64)
    _stream(os.path.join(dump_dir, "sen_vp_depthkernel.bin"), sen_vpRc, np.float64)
    _stream(os.path.join(dump_dir, "sen_rho_depthkernel.bin"), sen_rhoRc, np.float64)


def dump_depthkernel_ti(dump_dir, pvRc, Lsen_Gsc):
    os.makedirs(dump_dir, exist_ok=True)
    _stream(os.path.join(dump_dir, "pv_ti.bin"), pvRc, np.float64)
    _stream(os.path.join(dump_dir, "lsen_gsc_ti.bin"), Lsen_Gsc, np.float32)


def read_dump(path, shape, dtype):
    """A dump file as a Fortran-order array of the given shape."""
    return np.fromfile(path, dtype=dtype).reshape(shape, order="F")
