"""The reference arm of bench.py (`--impl reference`: the oracle timed on the
host cores) runs without a GPU: one JSON line with the contract's keys on
rank 0, and under torchrun the other ranks exit 0 without output."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--steps", "2", "--warmup", "1", "--cpu-cols-per-thread", "1",
        "--realisations", "1"]


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check(line):
    assert line["impl"] == "reference"
    assert line["metric"] == "kernel column-periods/s" and line["unit"] == "column-periods/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "config3"
    # the same config keys as our arm's line (the l2 note included)
    assert {"columns", "column_periods", "minthk", "parallelism", "l2"} <= set(line["config"])
    assert line["steps"] == 2 and line["ms_per_step"] > 0


def test_reference_arm_one_process():
    r = subprocess.run([sys.executable, "bench.py"] + ARGS, cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0])


def test_reference_arm_two_ranks_rank0_prints():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                        "--master-port", str(port), "bench.py", "--gpus", "2"] + ARGS,
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0])
    assert lines[0]["n_gpus"] == 2


def test_our_arm_fails_loudly_without_a_gpu():
    """No CPU fallback: without a device our arm exits non-zero and prints
    no measurement."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "bench.py", "--steps", "3", "--warmup", "3",
                        "--realisations", "1", "--no-cpu-baseline"], cwd=ROOT,
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode != 0
    assert _lines(r.stdout) == []


def test_accuracy_block_bookkeeping():
    """bench.py's accuracy block on CPU data: the oracle's own outputs as the
    'library' outputs give zero errors and full identity counts; a planted
    error in one column's kernels and one phase velocity shows up."""
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    from oracle import oracle as O
    from dazi_current_release_b200 import synthetic as S
    b = S.config3(realisations=1, columns=60)
    idx = bench.sample_columns(b, 6, 0)
    sb = bench.sub_batch(b, idx)
    for j, c in enumerate(idx):
        d, v, p = b.column(int(c))
        d2, v2, p2 = sb.column(j)
        assert np.array_equal(d, d2) and np.array_equal(v, v2) and np.array_equal(p, p2)
    ora = O.batch(sb.node_off, sb.depz, sb.vs, sb.per_off, sb.periods, sb.minthk)
    exact = O.batch_fd(sb.node_off, sb.depz, sb.vs, sb.per_off, sb.periods, sb.minthk,
                       exact=True)
    gpu = {k: ora[k].copy() for k in ("pv", "sen_vs", "sen_vp", "sen_rho", "lsen")}
    gpu["status"] = exact["status"].copy()
    acc = bench.accuracy_block(sb, gpu, ora, exact, dict(gpu))
    assert acc["pv_max_rel_err"] == 0.0 and acc["pv_bit_identical"] == sb.column_periods
    assert acc["status_equal_columns"] == sb.ncol
    assert acc["fundamental_mode_identity_columns"] == sb.ncol
    assert acc["lsen_worst_column_rel_l2"] == 0.0
    # the reference's FD kernels against the exact derivative: within its A/B gate
    for n, v in acc["adjoint_kernels_vs_exact_worst_column_rel_l2"].items():
        assert 0.0 < v <= 3e-3, (n, v)
    assert acc["plain_form"]["kernel_entries_bit_identical"] == acc["plain_form"]["kernel_entries"]
    # planted errors
    gpu["pv"][sb.per_off[2]] *= 1.0 + 3e-6
    gpu["sen_vs"][:] = exact["sen_vs"]
    acc = bench.accuracy_block(sb, gpu, ora, exact, None)
    assert 2e-6 < acc["pv_max_rel_err"] < 4e-6
    assert acc["fundamental_mode_identity_columns"] == sb.ncol - 1
    assert acc["adjoint_kernels_vs_exact_worst_column_rel_l2"]["sen_vs"] == 0.0
    assert "plain_form" not in acc
