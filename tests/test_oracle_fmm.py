"""The oracle of the reference's traveltime solver (oracle/fmm_oracle.c)
against the reference's own example run, and on closed-form cases.

- The Yunnan example (tests/golden/yunnan_fmm.npz): the forward traveltimes
  of the reference's last iteration, 20,877 source-receiver times from 1,469
  (period, source) fields, reproduced from that iteration's printed phase
  velocity maps.  The maps are printed to 1e-4 km/s, so the times can only
  agree to that resolution: |dt| <= 2.5e-3 s (max 1.7e-3 measured), median
  <= 3e-4 s, relative <= 2e-5.  A solver that differed in any step (first
  vs mixed order, source-grid refinement, the receiver interpolation, a
  source one refined cell off) is off by 0.03 s or more.
- A homogeneous sphere: times match the great-circle distance over the
  velocity to within one cell diagonal (the reference starts the front
  with the source cell's four corner times formed from angular distances,
  CalSurfG_parallel.f90:217-223, i.e. about zero) plus 0.5 % of the
  distance for the mixed-order scheme, 3 % for the first-order one (its
  error along the grid diagonals).
"""
import numpy as np
import pytest

import fmm_data


@pytest.fixture(scope="module")
def data(oracle):
    return fmm_data.load(oracle)


def test_yunnan_forward_times(oracle, data):
    d = data
    P = oracle.fmm_params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"])
    t = oracle.fmm_batch(P, d["pv"], d["inst_period"], d["scx"], d["scz"], d["rc_off"], d["rcx"],
                         d["rcz"])
    err = np.abs(t - d["t_forward"])
    print(f"max {err.max():.2e} s, median {np.median(err):.2e} s, "
          f"max rel {(err / d['t_forward']).max():.2e}")
    assert err.max() <= 2.5e-3
    assert np.median(err) <= 3e-4
    assert (err / d["t_forward"]).max() <= 2e-5


def _great_circle(x0, z0, x1, z1):
    c = np.sin(x0) * np.sin(x1) * np.cos(z0 - z1) + np.cos(x0) * np.cos(x1)
    return 6371.0 * np.arccos(np.clip(c, -1.0, 1.0))


@pytest.mark.parametrize("fom,rel", [(0, 0.03), (1, 0.005)])
def test_homogeneous_sphere(oracle, fom, rel):
    nnx, nnz = 61, 71
    gox, goz = np.float32(np.radians(60.0)), np.float32(np.radians(100.0))
    dnx = dnz = np.float32(np.radians(0.05))
    v = np.float32(3.5)
    veln = np.full((nnx, nnz), v, np.float32)
    scx = np.float32(gox + np.float32(30.3) * dnx)
    scz = np.float32(goz + np.float32(35.6) * dnz)
    ttn, st = oracle.fmm_travel(veln, gox, goz, dnx, dnz, scx, scz, fom=fom)
    assert (st == 0).all()
    ix, iz = np.meshgrid(np.arange(nnx), np.arange(nnz), indexing="ij")
    dist = _great_circle(np.float64(scx), np.float64(scz), gox + ix * np.float64(dnx),
                         goz + iz * np.float64(dnz))
    diag = 6371.0 * np.hypot(float(dnx), float(dnz) * np.sin(float(gox)))
    err = np.abs(ttn * v - dist)
    print(f"fom {fom}: max |t v - d| {err.max():.2f} km (cell diagonal {diag:.2f} km)")
    assert (err <= diag + rel * dist).all()
