"""The Yunnan data set of tests/golden/yunnan_fmm.npz as traveltime-solver
input: instances (one per source header, with its period), receivers in CSR,
coordinates converted as Main_Jt.f90:412-431 does (colatitude and longitude
in radians, float32), and the phase-velocity maps of the reference's last
iteration on the whole nx x ny grid (inner columns from the example's
printed maps; boundary columns, never updated by the inversion, from the
initial model through the oracle's surfdisp96)."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PI = np.float32(3.1415926535898)


def colat_rad(lat):
    return (np.float32(90.0) - np.asarray(lat, np.float32)) * PI / np.float32(180.0)


def lon_rad(lon):
    return np.asarray(lon, np.float32) * PI / np.float32(180.0)


def load(oracle):
    g = np.load(os.path.join(HERE, "golden", "yunnan_fmm.npz"))
    m = np.load(os.path.join(HERE, "golden", "yunnan_pv.npz"))
    vel, depz, periods = m["vel"], m["depz"], m["periods"]
    nx, ny, _ = vel.shape
    K = periods.size
    pv = np.array(oracle.depthkernel(vel, depz, periods, float(m["minthk"]), kernels=False)["pvRc"],
                  np.float64).reshape(nx * ny, K)
    inner = g["pv_inner_e4"].astype(np.float64) / 1e4          # (K, ny-2, nx-2)
    full = pv.reshape(ny, nx, K).copy()
    full[1:-1, 1:-1, :] = inner.transpose(1, 2, 0)
    st = g["station"]
    rc = st[g["rc_station"]]
    goxd, gozd, dvxd, dvzd = (float(v) for v in g["grid"])
    return {
        "nx": nx, "ny": ny, "K": K, "goxd": goxd, "gozd": gozd, "dvxd": dvxd, "dvzd": dvzd,
        "pv": np.asfortranarray(full.reshape(nx * ny, K)),
        "inst_period": g["src_period"].astype(np.int32) - 1,
        "scx": colat_rad(g["src_lat"]), "scz": lon_rad(g["src_lon"]),
        "rc_off": g["rc_off"].astype(np.int64),
        "rcx": colat_rad(rc[:, 0]), "rcz": lon_rad(rc[:, 1]),
        "t_forward": g["t_forward"].astype(np.float64),
    }
