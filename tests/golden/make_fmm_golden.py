"""Generate tests/golden/yunnan_fmm.npz from the reference's own example run.

Reads, in the reference checkout, examples/test4_Yunnan/smooth/:
  - China_YN_Rayleigh_RS_5-40s.dat: the data set, read as
    code/src_inv_iso_joint/Main_Jt.f90:394-440 reads it ('#' lines are
    sources with their period index, the other lines their receivers);
  - phaseV_FWD.dat: the phase-velocity maps of the inner (nx-2)*(ny-2)
    columns at 36 periods (WTPeriodPhaseV, Main_Jt.f90:2019-2038, f10.4),
    written after the last iteration from the maps of its G computation;
  - Traveltime_use_10th.dat: the forward traveltimes of that same
    computation (T_forward, Main_Jt.f90:727-737), i.e. FMM traveltimes
    (CalSurfG_parallel.f90:2148-2335) through those maps.
The boundary columns of the maps are not printed; the inversion never
updates them (Main_Jt.f90:1258-1285 updates vsf(i+1, j+1, k) only), so they
are the initial model's (examples/.../MOD, stored in yunnan_pv.npz) and the
tests compute them with the oracle's phase velocities.

Usage: python tests/golden/make_fmm_golden.py REFERENCE_ROOT
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

if len(sys.argv) != 2:
    sys.exit(__doc__)
base = os.path.join(sys.argv[1], "examples", "test4_Yunnan", "smooth")
nx, ny, K = 38, 42, 36
src_lat, src_lon, src_per, rc_off, rc_lat, rc_lon = [], [], [], [0], [], []
with open(os.path.join(base, "China_YN_Rayleigh_RS_5-40s.dat")) as f:
    for line in f:
        t = line.split()
        if not t:
            continue
        if line.startswith("#"):
            lat, lon, per, wave, igr = t[1], t[2], int(t[3]), int(t[4]), int(t[5])
            assert (wave, igr) == (2, 0)
            src_lat.append(np.float32(lat))
            src_lon.append(np.float32(lon))
            src_per.append(per)
            rc_off.append(rc_off[-1])
        else:
            rc_lat.append(np.float32(t[0]))
            rc_lon.append(np.float32(t[1]))
            rc_off[-1] += 1
fwd = np.loadtxt(os.path.join(base, "phaseV_FWD.dat"))
assert fwd.shape == ((nx - 2) * (ny - 2) * K, 4)
pv_e4 = np.rint(fwd[:, 3] * 1e4).astype(np.uint16).reshape(K, ny - 2, nx - 2)
tt = np.loadtxt(os.path.join(base, "Traveltime_use_10th.dat"), skiprows=1)
assert tt.shape[0] == rc_off[-1]
# stations as a table plus indices (the receivers repeat)
st, inv = np.unique(np.stack([rc_lat, rc_lon], 1), axis=0, return_inverse=True)
np.savez_compressed(os.path.join(HERE, "yunnan_fmm.npz"),
                    src_lat=np.array(src_lat, np.float32), src_lon=np.array(src_lon, np.float32),
                    src_period=np.array(src_per, np.int16), rc_off=np.array(rc_off, np.int32),
                    station=st.astype(np.float32), rc_station=inv.astype(np.int16).ravel(),
                    pv_inner_e4=pv_e4, t_forward=tt[:, 2].astype(np.float32),
                    grid=np.array([29.0, 98.0, 0.25, 0.25], np.float32))
print(f"wrote yunnan_fmm.npz: {len(src_lat)} sources, {rc_off[-1]} receivers "
      f"({st.shape[0]} stations)")
