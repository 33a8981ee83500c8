"""Multi-GPU host logic on the CPU: shard boundaries, CSR slicing and the
gather of the outputs (size exchange + point-to-point receives into slices
of the destination's arrays), run as world-size-2 (and 3) gloo process
groups.
The per-shard computation is the oracle here (the library needs a GPU);
the test checks that the sharded, gathered result equals the oracle run on
the whole batch in one process."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dazi_current_release_b200 import shard
from dazi_current_release_b200 import synthetic as S


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_bounds_cover_and_balance():
    rng = np.random.default_rng(0)
    work = rng.integers(10, 2000, 1000)
    for world in (1, 2, 3, 8):
        b = shard.shard_bounds(work, world)
        assert b[0] == 0 and b[-1] == work.size and (np.diff(b) >= 1).all()
        loads = [work[b[r]:b[r + 1]].sum() for r in range(world)]
        assert max(loads) <= work.sum() / world + work.max()
    # more ranks than columns: empty shards at the end, still a cover
    b = shard.shard_bounds([5, 5], 4)
    assert b[0] == 0 and b[-1] == 2 and (np.diff(b) >= 0).all()


def test_slice_rebases_offsets():
    b = S.config3(realisations=1, columns=20)
    part = shard.slice_batch(b.node_off, b.depz, b.vs, b.per_off, b.periods, 5, 9)
    assert part["node_off"][0] == 0 and part["per_off"][0] == 0
    for i, c in enumerate(range(5, 9)):
        d, v, p = b.column(c)
        a0, a1 = part["node_off"][i], part["node_off"][i + 1]
        np.testing.assert_array_equal(part["depz"][a0:a1], d)
        np.testing.assert_array_equal(part["vs"][a0:a1], v)
        np.testing.assert_array_equal(part["periods"][part["per_off"][i]:part["per_off"][i + 1]], p)


def _oracle_compute(part, minthk, form):
    from oracle import oracle as O
    r = O.batch(part["node_off"], part["depz"], part["vs"], part["per_off"], part["periods"],
                minthk, nthreads=2)
    pv = r["pv"]
    st = np.zeros(part["node_off"].size - 1, np.int32)
    for c in range(st.size):
        seg = pv[part["per_off"][c]:part["per_off"][c + 1]]
        if (seg <= 0).any():
            st[c] = int(np.argmin(seg > 0)) + 1
    return dict(pv=pv, sen_vs=r["sen_vs"], sen_vp=r["sen_vp"], sen_rho=r["sen_rho"],
                lsen=r["lsen"], status=st)


def _worker(rank, world, port, path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        b = S.config3(realisations=1, columns=8, base_seed=1000)
        out = shard.run_sharded(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk,
                                compute=_oracle_compute)
        if rank == 0:
            np.savez(path, **{k: (v.numpy() if hasattr(v, "numpy") else v)
                              for k, v in out.items() if v is not None})
        else:
            assert out is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_run_equals_single_process(tmp_path, world):
    path = str(tmp_path / "out.npz")
    mp.start_processes(_worker, args=(world, _free_port(), path), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(path)
    b = S.config3(realisations=1, columns=8, base_seed=1000)
    ref = _oracle_compute(dict(node_off=b.node_off, depz=b.depz, vs=b.vs, per_off=b.per_off,
                               periods=b.periods), b.minthk, 1)
    for k in ("pv", "sen_vs", "sen_vp", "sen_rho", "lsen", "status"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def _gather_worker(rank, world, port, path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        # uneven blocks, one rank with empty ones, two dtypes
        n = [5, 0, 3][rank]
        blocks = {"a": torch.arange(n, dtype=torch.float64) + 100 * rank,
                  "b": torch.full((2 * n,), rank, dtype=torch.int32)}
        out = shard.gather_blocks(blocks, dst=world - 1)
        if rank == world - 1:
            np.savez(path, a=out["a"].numpy(), b=out["b"].numpy())
        else:
            assert out is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gather_blocks_concatenates_in_rank_order(tmp_path):
    path = str(tmp_path / "g.npz")
    mp.start_processes(_gather_worker, args=(3, _free_port(), path), nprocs=3, join=True,
                       start_method="spawn")
    g = np.load(path)
    np.testing.assert_array_equal(g["a"], np.concatenate([np.arange(5.0), 200 + np.arange(3.0)]))
    np.testing.assert_array_equal(g["b"], np.array([0] * 10 + [2] * 6, np.int32))
