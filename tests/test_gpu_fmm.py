"""The GPU traveltime solver (dazi_fmm_batch, dazi_fmm_batch_dev,
dazi_fmm_times) against the oracle (oracle/fmm_oracle.c):
- the whole Yunnan example (1,469 (period, source) fields, 20,877 receiver
  times): times bit-identical to the oracle's, and within the printed
  maps' resolution of the reference run's own forward times (2.5e-3 s);
  the coarse fields of every 25th instance bit-identical;
- seeded synthetic data sets reaching the solver's branches, with and
  without source-grid refinement and with both upwind schemes, and a large
  grid whose narrow bands outgrow the shared-memory part of the heap;
- the device-pointer entry equals the host entry, and the Fortran-shaped
  entry (the reference's source and receiver tables) equals the batch;
- a source outside the grid, a narrow band beyond its capacity and a source
  whose refined sweep ends before any coarse node are reported errors."""
import ctypes

import numpy as np
import pytest

import fmm_data
from dazi_current_release_b200 import _lib
from dazi_current_release_b200 import fmm

pytestmark = pytest.mark.gpu


def _params(d, **kw):
    return fmm.params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"], **kw)


@pytest.fixture(scope="module")
def yunnan(oracle):
    return fmm_data.load(oracle)


def test_yunnan_times_bit_identical(oracle, yunnan):
    d = yunnan
    P = oracle.fmm_params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"])
    ref = oracle.fmm_batch(P, *fmm_data.args(d))
    got = fmm.travel_times(_params(d), *fmm_data.args(d))
    np.testing.assert_array_equal(got, ref)
    err = np.abs(got - d["t_forward"])
    print(f"{got.size} times equal to the oracle's; vs the reference run max {err.max():.2e} s")
    assert err.max() <= 2.5e-3


def test_yunnan_fields_bit_identical(oracle, yunnan):
    d = fmm_data.subset(yunnan, np.arange(0, yunnan["inst_period"].size, 25))
    P = oracle.fmm_params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"])
    t0, f0 = oracle.fmm_batch(P, *fmm_data.args(d), fields=True)
    t1, f1 = fmm.travel_times(_params(d), *fmm_data.args(d), fields=True)
    np.testing.assert_array_equal(t1, t0)
    np.testing.assert_array_equal(f1, f0)


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
@pytest.mark.parametrize("kw", [{}, {"asgr": 0}, {"fom": 0}, {"asgr": 0, "fom": 0}])
def test_synthetic_bit_identical(oracle, seed, kw):
    d = fmm_data.synthetic(seed)
    P = oracle.fmm_params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"], **kw)
    t0, f0 = oracle.fmm_batch(P, *fmm_data.args(d), fields=True)
    t1, f1 = fmm.travel_times(_params(d, **kw), *fmm_data.args(d), fields=True)
    np.testing.assert_array_equal(t1, t0)
    np.testing.assert_array_equal(f1, f0)


def test_large_band_bit_identical(oracle):
    d = fmm_data.big_case()
    P = oracle.fmm_params(d["nx"], d["ny"], d["goxd"], d["gozd"], d["dvxd"], d["dvzd"])
    t0, f0 = oracle.fmm_batch(P, *fmm_data.args(d), fields=True)
    t1, f1 = fmm.travel_times(_params(d), *fmm_data.args(d), fields=True)
    np.testing.assert_array_equal(t1, t0)
    np.testing.assert_array_equal(f1, f0)


def test_device_entry_equals_host_entry(yunnan):
    torch = pytest.importorskip("torch")
    d = fmm_data.subset(yunnan, np.arange(0, yunnan["inst_period"].size, 7))
    host = fmm.travel_times(_params(d), *fmm_data.args(d))
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    pv = t(np.asfortranarray(d["pv"]).T.copy().ravel())       # column-major (nx*ny, nper)
    got = fmm.travel_times_dev(_params(d), pv, t(d["inst_period"]), t(d["scx"]), t(d["scz"]),
                               t(d["rc_off"]), t(d["rcx"]), t(d["rcz"]))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), host)


def test_fortran_entry_equals_batch(yunnan):
    """dazi_fmm_times on the reference's own tables (scxf(nsrc, kmax), rcxf
    (nrc, nsrc, kmax), nrc1, nsrc1, periods) built from the data set."""
    d = yunnan
    K = d["K"]
    per = d["inst_period"]
    nsrc1 = np.bincount(per, minlength=K).astype(np.int32)
    NS, NR = int(nsrc1.max()), int(np.diff(d["rc_off"]).max())
    scxf = np.zeros((NS, K), np.float32, order="F")
    sczf = np.zeros_like(scxf)
    periods = np.zeros((NS, K), np.int32, order="F")
    nrc1 = np.zeros((NS, K), np.int32, order="F")
    rcxf = np.zeros((NR, NS, K), np.float32, order="F")
    rczf = np.zeros_like(rcxf)
    fill = np.zeros(K, int)
    order = []
    for s in range(per.size):      # the data file lists the periods in order
        k = per[s]
        j = fill[k]
        fill[k] += 1
        scxf[j, k], sczf[j, k], periods[j, k] = d["scx"][s], d["scz"][s], k + 1
        a, b = d["rc_off"][s], d["rc_off"][s + 1]
        nrc1[j, k] = b - a
        rcxf[:b - a, j, k], rczf[:b - a, j, k] = d["rcx"][a:b], d["rcz"][a:b]
        order.append((k, j, s))
    order.sort()
    idx = np.concatenate([np.arange(d["rc_off"][s], d["rc_off"][s + 1]) for _, _, s in order])
    dall = int(d["rc_off"][-1])
    dsurf = np.zeros(dall, np.float32)
    L = _lib.load()
    I = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    F = lambda v: ctypes.byref(ctypes.c_float(v))  # noqa: E731
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))  # noqa: E731
    pv = np.asfortranarray(d["pv"])
    rc = L.dazi_fmm_times(I(d["nx"]), I(d["ny"]), I(K), I(NS), I(NR), I(pv.shape[1]),
                          P(pv, ctypes.c_double), P(periods, ctypes.c_int), P(nsrc1, ctypes.c_int),
                          P(nrc1, ctypes.c_int), P(scxf, ctypes.c_float), P(sczf, ctypes.c_float),
                          P(rcxf, ctypes.c_float), P(rczf, ctypes.c_float), F(d["goxd"]), F(d["gozd"]),
                          F(d["dvxd"]), F(d["dvzd"]), ctypes.byref(ctypes.c_longlong(dall)),
                          P(dsurf, ctypes.c_float))
    assert rc == 0, L.dazi_dk_last_error()
    ref = fmm.travel_times(_params(d), *fmm_data.args(d))
    np.testing.assert_array_equal(dsurf, ref[idx])


def test_errors():
    d = fmm_data.synthetic(0)
    lat1 = d["goxd"] - d["dvxd"] * (d["nx"] - 3)

    def one(lat, lon, **kw):
        e = fmm_data.subset(d, np.array([0]))
        e["scx"], e["scz"] = fmm_data.colat_rad([lat]), fmm_data.lon_rad([lon])
        return fmm.travel_times(_params(e, **kw), *fmm_data.args(e))

    with pytest.raises(_lib.DaziError) as ei:
        one(d["goxd"] + 0.3, d["gozd"] + 1.0)
    assert ei.value.code == _lib.DAZI_ERR_BADARG
    with pytest.raises(_lib.DaziError) as ei:
        one(lat1 + 0.003, d["gozd"] + 1.025)
    assert ei.value.code == _lib.DAZI_ERR_MODEL
    with pytest.raises(_lib.DaziError) as ei:
        one(d["goxd"] - 1.0, d["gozd"] + 1.0, snb=0.002)
    assert ei.value.code == _lib.DAZI_ERR_LIMITS
    # the library stays usable
    t = one(d["goxd"] - 1.0, d["gozd"] + 1.0)
    assert np.isfinite(t).all()
