"""The reference arm of bench.py (`--impl reference`: the oracle timed on the
host cores) runs without a GPU: one JSON line with the contract's keys on
rank 0, and under torchrun the other ranks exit 0 without output."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "1", "--cpu-sample-s", "0.3",
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
