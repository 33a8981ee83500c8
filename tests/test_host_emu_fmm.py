"""The library's traveltime device code (csrc/fmm_device.cuh), compiled for
the host by tests/host_emu and driven as the library drives it, against the
oracle (oracle/fmm_oracle.c) on the CPU: bit-identical receiver times and
coarse fields
- on every 10th instance of the Yunnan example (147 of 1,469),
- on seeded synthetic data sets that reach the solver's branches (sources
  on nodes and in the corner cells, refined boxes cut by the model's sides,
  receivers in and next to the source's cell), with and without source-grid
  refinement and with both upwind schemes,
- on a large grid whose narrow bands outgrow the heap part the GPU keeps
  in shared memory;
and the same error where the reference's field is undefined (a source in the
last cell before the right side) or a source lies outside the grid.  The
same code runs on the GPU (tests/test_gpu_fmm.py)."""
import numpy as np
import pytest

import fmm_data
from host_emu import emu


def _both(oracle, d, **kw):
    P = oracle.fmm_params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"], **kw)
    ref = oracle.fmm_batch(P, *fmm_data.args(d), fields=True)
    got = emu.fmm_batch(P, *fmm_data.args(d), fields=True)
    return ref, got


def test_yunnan_subset_bit_identical(oracle):
    d = fmm_data.load(oracle)
    d = fmm_data.subset(d, np.arange(0, d["inst_period"].size, 10))
    (t0, f0), (t1, f1) = _both(oracle, d)
    np.testing.assert_array_equal(t1, t0)
    np.testing.assert_array_equal(f1, f0)
    assert np.abs(t1 - d["t_forward"]).max() <= 2.5e-3


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("kw", [{}, {"asgr": 0}, {"fom": 0}, {"asgr": 0, "fom": 0}])
def test_synthetic_bit_identical(oracle, seed, kw):
    d = fmm_data.synthetic(seed)
    (t0, f0), (t1, f1) = _both(oracle, d, **kw)
    np.testing.assert_array_equal(t1, t0)
    np.testing.assert_array_equal(f1, f0)


def test_large_band_bit_identical(oracle):
    (t0, f0), (t1, f1) = _both(oracle, fmm_data.big_case())
    np.testing.assert_array_equal(t1, t0)
    np.testing.assert_array_equal(f1, f0)


def _one_source(d, lat, lon):
    d = fmm_data.subset(d, np.array([0]))
    d["scx"] = fmm_data.colat_rad([lat])
    d["scz"] = fmm_data.lon_rad([lon])
    return d


def test_undefined_field_and_outside_source_are_errors(oracle):
    d = fmm_data.synthetic(0)
    lat1 = d["goxd"] - d["dvxd"] * (d["nx"] - 3)
    # half a refined cell from the bottom (largest colatitude) side and
    # midway between coarse columns: the refined sweep stops at once, with
    # no coarse node in its band
    e = _one_source(d, lat1 + 0.003, d["gozd"] + 1.025)
    with pytest.raises(RuntimeError, match="error -5"):
        _both(oracle, e)
    with pytest.raises(RuntimeError, match="instance error 5"):
        P = oracle.fmm_params(e["nx"], e["ny"], e["goxd"], e["gozd"], e["dvxd"], e["dvzd"])
        emu.fmm_batch(P, *fmm_data.args(e))
    o = _one_source(d, d["goxd"] + 0.3, d["gozd"] + 1.0)
    P = oracle.fmm_params(o["nx"], o["ny"], o["goxd"], o["gozd"], o["dvxd"], o["dvzd"])
    with pytest.raises(RuntimeError, match="error -1"):
        oracle.fmm_batch(P, *fmm_data.args(o))
    with pytest.raises(RuntimeError, match="emu fmm_batch: -1"):
        emu.fmm_batch(P, *fmm_data.args(o))
