"""The library's root search (root_kernel and its state machine), compiled
for the host by tests/host_emu, against the oracle of surfdisp96 on the CPU,
and its FP32 coarse scan (FP32 sign of the secular function on the getsol
scan steps, FP64 re-evaluation below the trust threshold and at both ends
of every bracket) against the all-FP64 scan: identical roots and statuses,
bit for bit."""
import numpy as np

from dazi_current_release_b200 import synthetic as S
from edge_models import _batch, _random_columns
from host_emu import emu


def _cases():
    b = S.config3(realisations=1, columns=240, base_seed=1000)
    yield "uneven", (b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    yield "random", (*_batch(_random_columns(120, seed=3)), 2.0)


def test_fp32_scan_gives_the_fp64_roots():
    for name, args in _cases():
        rc64, pv64, st64, _ = emu.root_batch(*args, scan32=False)
        rc32, pv32, st32, _ = emu.root_batch(*args, scan32=True)
        assert rc64 == 0 and rc32 == 0
        np.testing.assert_array_equal(pv32, pv64, err_msg=name)
        np.testing.assert_array_equal(st32, st64, err_msg=name)


def test_root_search_matches_oracle_on_uneven_columns(oracle):
    b = S.config3(realisations=1, columns=240, base_seed=1000)
    rc, pv, st, _ = emu.root_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk)
    ref = oracle.batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                       kernels=False, lsen=True)
    assert rc == 0
    np.testing.assert_array_equal(pv[:ref["pv"].size], ref["pv"])
