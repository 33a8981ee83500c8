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


def synthetic(seed, nx=20, ny=24, nper=3, nsrc=12, nrc=15):
    """A seeded data set on an nx x ny grid (first inner vertex 30 N, 100 E,
    0.25 deg) with smooth random maps (2.8-3.8 km/s) and the cases the
    reference's solver branches on: sources on grid nodes, on the last node
    and in the corner cells (refined boxes cut by the model's sides),
    receivers in the source's cell and next to it (srtimes' near-source
    formula), receivers on the grid's last row and column."""
    rng = np.random.default_rng(seed)
    goxd, gozd, dv = 30.0, 100.0, 0.25
    lat0, lon0 = goxd, gozd                       # first propagation node
    lat1, lon1 = goxd - dv * (nx - 3), gozd + dv * (ny - 3)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    pv = np.zeros((nx * ny, nper))
    for k in range(nper):
        a, b, c = rng.uniform(0.5, 2.0, 3)
        m = 3.3 + 0.25 * np.sin(a * ii / 3.0 + c) * np.cos(b * jj / 4.0) + 0.05 * rng.standard_normal((nx, ny))
        pv[:, k] = np.float32(m).T.ravel()         # x (latitude) index fastest
    # the reference cannot start from the last cells before the right or
    # bottom side (its refined sweep stops at that side before reaching a
    # coarse node) nor from the last node (srtimes reads past the grid),
    # so the sources there sit 1.5 and 2.5 coarse cells inside
    slat = np.concatenate([rng.uniform(lat1 + 0.11, lat0, nsrc - 5),
                           [lat0, lat1 + 0.075, lat0 - 0.05, lat1 + 0.125, lat0 - dv * 3]])
    slon = np.concatenate([rng.uniform(lon0, lon1 - 0.11, nsrc - 5),
                           [lon0, lon1 - 0.075, lon0 + 0.05, lon1 - 0.125, lon0 + dv * 4]])
    slat[:3], slon[:3] = np.round(slat[:3] / 0.05) * 0.05, np.round(slon[:3] / 0.05) * 0.05
    inst_p, sx, sz, rx, rz, off = [], [], [], [], [], [0]
    for s in range(nsrc):
        inst_p.append(s % nper)
        sx.append(slat[s]); sz.append(slon[s])
        la = list(rng.uniform(lat1, lat0, nrc - 4)) + [slat[s] - 0.003, slat[s] + 0.01, lat1, lat0]
        lo = list(rng.uniform(lon0, lon1, nrc - 4)) + [slon[s] + 0.004, slon[s] - 0.02, lon1, lon0]
        la = np.clip(la, lat1 + 1e-4, lat0); lo = np.clip(lo, lon0, lon1 - 1e-4)
        rx += list(la); rz += list(lo)
        off.append(off[-1] + nrc)
    return {"nx": nx, "ny": ny, "goxd": goxd, "gozd": gozd, "dvxd": dv, "dvzd": dv, "pv": pv,
            "inst_period": np.array(inst_p, np.int32), "scx": colat_rad(sx), "scz": lon_rad(sz),
            "rc_off": np.array(off, np.int64), "rcx": colat_rad(rx), "rcz": lon_rad(rz)}


def big_case():
    """Two sources on a 1136 x 1136 propagation grid: narrow bands of more
    than 1,535 nodes, beyond the heap positions a warp keeps in shared
    memory on the GPU."""
    return subset(synthetic(5, nx=230, ny=230, nper=1, nsrc=6, nrc=6), np.array([0, 4]))


def subset(d, sel):
    """The instances sel of a data set, with their receivers."""
    off = d["rc_off"]
    ro = np.concatenate([[0], np.cumsum(off[sel + 1] - off[sel])]).astype(np.int64)
    idx = np.concatenate([np.arange(off[s], off[s + 1]) for s in sel])
    out = dict(d)
    out.update(inst_period=d["inst_period"][sel], scx=d["scx"][sel], scz=d["scz"][sel], rc_off=ro,
               rcx=d["rcx"][idx], rcz=d["rcz"][idx])
    if "t_forward" in d:
        out["t_forward"] = d["t_forward"][idx]
    return out


def args(d):
    return (d["pv"], d["inst_period"], d["scx"], d["scz"], d["rc_off"], d["rcx"], d["rcz"])
