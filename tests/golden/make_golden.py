"""Generate tests/golden/yunnan_pv.npz from the reference's own example files.

Reads (in the reference checkout) examples/test4_Yunnan/voro/MOD (initial Vs
model, read as in code/src_inv_iso_joint/Main_Jt.f90:518-528),
examples/test4_Yunnan/voro/para.in (minthk = 4 sublayers, periods 5..40 s)
and the two golden phase-velocity maps written by WTPeriodPhaseV
(Main_Jt.f90:2019-2038):
  examples/test4_Yunnan_legacy_old_para/voro/period_phaseVMOD.dat
  examples/test4_Yunnan/voro/period_phaseVMOD.dat
Both hold surfdisp96 phase velocities of the inner (nx-2)*(ny-2) columns at
36 periods, printed with f10.4.  They are stored as integers (value * 1e4).

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit(__doc__)
ref = sys.argv[1]   # the reference checkout (the root of the DAzi project)
base = os.path.join(ref, "examples", "test4_Yunnan", "voro")
legacy = os.path.join(ref, "examples", "test4_Yunnan_legacy_old_para", "voro")
nx, ny, nz = 38, 42, 18
with open(os.path.join(base, "MOD")) as f:
    depz = np.array(f.readline().split(), np.float32)
    vals = np.array(f.read().split(), np.float32)
assert depz.size == nz and vals.size == nx * ny * nz
vel = np.zeros((nx, ny, nz), np.float32, order="F")
i = 0
for k in range(nz):
    for j in range(ny):
        vel[:, j, k] = vals[i:i + nx]
        i += nx
periods = np.arange(5, 41, dtype=np.float64)


def load_pv(path):
    g = np.loadtxt(path)
    assert g.shape == ((nx - 2) * (ny - 2) * periods.size, 4)
    assert np.allclose(np.unique(g[:, 2]), periods)
    return np.rint(g[:, 3] * 1e4).astype(np.uint16)


np.savez_compressed(
    os.path.join(os.path.dirname(os.path.abspath(__file__)), "yunnan_pv.npz"),
    vel=vel, depz=depz, periods=periods, minthk=np.float32(4.0),
    nx=nx, ny=ny, nz=nz,
    pv_legacy_e4=load_pv(os.path.join(legacy, "period_phaseVMOD.dat")),
    pv_current_e4=load_pv(os.path.join(base, "period_phaseVMOD.dat")))
print("wrote yunnan_pv.npz")
