"""The reference's output formats: Fortran F edit descriptors, the
period_phaseVMOD.dat layout of WTPeriodPhaseV (checked against the
reference's own golden output values), and the unformatted dumps."""
import numpy as np

from conftest import inner_columns
from dazi_current_release_b200 import formats


def test_fortran_f():
    assert formats.fortran_f(0.5, 10, 4) == "    0.5000"
    assert formats.fortran_f(-3.14159, 10, 5) == "  -3.14159"
    assert formats.fortran_f(123456789.0, 10, 4) == "*" * 10


def test_period_phasev_reproduces_golden_values(oracle, yunnan, tmp_path):
    y = yunnan
    nx, ny = int(y["nx"]), int(y["ny"])
    r = oracle.depthkernel(y["vel"], y["depz"], y["periods"], float(y["minthk"]), kernels=False)
    K = y["periods"].size
    inner = np.stack([inner_columns(r["pvRc"][:, k:k + 1], nx, ny) for k in range(K)], axis=1)
    p = tmp_path / "period_phaseVMOD.dat"
    formats.write_period_phasev(p, nx, ny, 20.0, 100.0, 0.1, 0.1, y["periods"], inner)
    lines = p.read_text().splitlines()
    assert len(lines) == K * (nx - 2) * (ny - 2)
    assert all(len(s) == 40 for s in lines)
    pv = np.array([float(s[30:40]) for s in lines])
    np.testing.assert_array_equal(np.rint(pv * 1e4).astype(np.int64),
                                  y["pv_legacy_e4"].astype(np.int64))
    per = np.array([float(s[20:30]) for s in lines]).reshape(K, -1)
    np.testing.assert_allclose(per[:, 0], y["periods"], atol=5e-5)


def test_dumps_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    pv = np.asfortranarray(rng.standard_normal((6, 4)))
    s = [np.asfortranarray(rng.standard_normal((6, 4, 5))) for _ in range(3)]
    ls = np.asfortranarray(rng.standard_normal((6, 4, 4)).astype(np.float32))
    formats.dump_depthkernel(tmp_path, pv, *s)
    formats.dump_depthkernel_ti(tmp_path, pv, ls)
    np.testing.assert_array_equal(formats.read_dump(tmp_path / "pv_depthkernel.bin", (6, 4), np.float64), pv)
    np.testing.assert_array_equal(
        formats.read_dump(tmp_path / "sen_rho_depthkernel.bin", (6, 4, 5), np.float64), s[2])
    np.testing.assert_array_equal(
        formats.read_dump(tmp_path / "lsen_gsc_ti.bin", (6, 4, 4), np.float32), ls)
    assert (tmp_path / "pv_depthkernel.bin").stat().st_size == 6 * 4 * 8
