#!/usr/bin/env python
"""Benchmark of the depth-kernel stage: kernel column-periods per second.

One column-period = the Rayleigh phase velocity c(T) of one column plus its
Vs-type kernels (dc/dVs, dc/dVp, dc/drho at every node) plus its Gc/Gs kernel
(Lsen_Gsc at every depth interval).  A "step" is one pass of the stage over
the whole workload (one phase-velocity pass feeds both kernel kinds).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload config3]
                    [--form plain|adjoint] [--impl ours|reference]

Default workload: the uneven batch, 100 realisations x 2500 columns (10-60
layers, 8-40 periods each, sediments and low-velocity zones), through the
ragged batch entries dazi_dk_batch_dev / dazi_dk_batch.  The grid workloads
(config0/1/2/4: one depth grid for all columns) go through
dazi_dk_fused_dev / dazi_dk_fused.

value      device-timed throughput of the chosen form (--form, default the
           adjoint form; --root reference: the reference's point sequence, or
           brent: each period's bracket refined by Brent's method,
           DAZI_FORM_FAST_ROOT; the other one is timed beside it in
           root_search) on the whole batch, inputs resident in HBM: a plan
           (dazi_dk_plan_*: structure bound once, kernel variants autotuned,
           each step one CUDA-graph launch) on torch's stream, CUDA events per
           step, L2 flushed between steps outside the timed events; the
           per-call entry dazi_dk_batch_dev is timed beside it (per_call)
same_columns  both forms timed the same way on the first --plain-cols
           columns (the plain perturb-and-recompute form runs 1 + 6 nz root
           searches per column and would take minutes on the whole batch)
e2e        the same stage through the host C-ABI entry with pinned host
           buffers: host->device inputs and device->host outputs every step
roofline   FP64 CUDA-core bound of the dominant kernel (per-phase CUDA events
           inside the library): algorithmic flops = root search 180 per layer
           of each of the reference's secular evaluations (E_ref, counted by a
           run of the reference's search), adjoint and Gc/Gs sweeps 180 x 2 per
           layer item; pipe_frac from the FP64 operations ncu counts as executed
           (profiles/kernel_work.json); peak the FP64 FMA rate measured live by
           dazi_dk_fp64_peak
accuracy   errors on the cpu_baseline's sampled columns against the oracle
cpu_baseline  the CPU oracle (C restatement of the reference Fortran, OpenMP
           over columns) on a bounded sample of the same workload

Multi-GPU (torchrun): columns are independent, so every rank runs the same
per-GPU workload with no data-path collective (weak scaling); the step time
is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FLOP_PER_LAYER_EVAL = 180   # hand count of dltar4's FP64 arithmetic per layer of one secular
                             # evaluation (sqrt and division as one, transcendentals not counted)
SWEEP_FWD_EQUIV = 2          # forward-equivalent sweeps per layer item of the adjoint and of the
                             # Gc/Gs kernel (2 + 2 = the + 4 of the whole-step count)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--workload", default="config3")
    p.add_argument("--realisations", type=int, default=100,
                   help="ragged workload: realisations of 2500 columns per GPU")
    p.add_argument("--plain-cols", type=int, default=25000,
                   help="ragged workload: columns the plain form is timed on")
    p.add_argument("--form", default="adjoint", choices=["plain", "adjoint"])
    p.add_argument("--root", default="reference", choices=["brent", "reference"],
                   help="adjoint form: refine each period's bracket by Brent's method "
                        "(DAZI_FORM_FAST_ROOT) or by the reference's nevill()")
    p.add_argument("--no-other-form", action="store_true")
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-cols-per-thread", type=int, default=CPU_COLS_PER_THREAD,
                   help="uneven workload: columns per host thread in each CPU sample")
    p.add_argument("--cpu-sample-s", type=float, default=15.0,
                   help="grid workloads: seconds of CPU work in the cpu_baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fmm", action="store_true",
                   help="skip the traveltime-solver measurement (fmm block)")
    p.add_argument("--no-lsmr", action="store_true",
                   help="skip the LSMR solver measurement (lsmr block)")
    p.add_argument("--full-stack", action="store_true",
                   help="adjoint and Gc/Gs sweeps over the whole layer stack (no depth cut)")
    return p.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if args.impl == "ours":
            torch.cuda.set_device(local)
        # the reference arm runs on the host cores: no device, gloo
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=300))
    return ws, rank, local


def load_case(name):
    from dazi_current_release_b200 import synthetic as S
    return S.GRID_CONFIGS[name]()


def load_ragged(args, rank):
    """The uneven-column batch (per rank its own realisations: weak scaling)."""
    from dazi_current_release_b200 import synthetic as S
    return S.config3(realisations=args.realisations, base_seed=1000 + 100000 * rank)


CPU_COLS_PER_THREAD = 8   # default CPU sample: uneven columns per host thread (load-balanced)


def sample_columns(b, n, seed):
    """n columns drawn without replacement, seeded, from the whole batch
    (every realisation), in batch order."""
    return np.sort(np.random.default_rng(seed).choice(b.ncol, min(n, b.ncol), replace=False))


def sub_batch(b, idx):
    """The CSR batch of the columns idx."""
    from dazi_current_release_b200 import synthetic as S
    nz = np.diff(b.node_off)[idx]
    K = np.diff(b.per_off)[idx]
    cat = lambda arr, off: np.concatenate([arr[off[c]:off[c + 1]] for c in idx])  # noqa: E731
    return S.RaggedBatch(np.concatenate([[0], np.cumsum(nz)]).astype(np.int64),
                         cat(b.depz, b.node_off), cat(b.vs, b.node_off),
                         np.concatenate([[0], np.cumsum(K)]).astype(np.int64),
                         cat(b.periods, b.per_off), b.minthk)


def ragged_cpu_baseline(b, seed=0, cores=None, per_thread=CPU_COLS_PER_THREAD):
    """Oracle of the reference stage (depthkernel FD + depthkernelTI per
    column, OpenMP over columns) on a seeded sample of per_thread columns per
    host thread drawn from the whole batch; returns (the cpu_baseline entry,
    the sampled column indices, the sub-batch, the oracle outputs)."""
    from oracle import oracle as O
    cores = cores or os.cpu_count() or 1
    idx = sample_columns(b, per_thread * cores, seed)
    sb = sub_batch(b, idx)
    t0 = time.perf_counter()
    out = O.batch(sb.node_off, sb.depz, sb.vs, sb.per_off, sb.periods, sb.minthk, nthreads=cores)
    dt = time.perf_counter() - t0
    cp = sb.column_periods
    cb = {"value": cp / dt, "unit": "column-periods/s", "cores": cores, "kind": "port",
          "sample": f"{idx.size} seeded columns (seed {seed}) drawn from the {b.ncol} of the "
                    f"batch ({cp} column-periods), oracle of depthkernel (FD: 1+6nz "
                    f"surfdisp96 per column) + depthkernelTI at -O3, {dt:.1f} s on {cores} "
                    f"threads"}
    return cb, idx, sb, out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def _cpu_stage(O, flat, vp, rho, case, n, cores):
    """The reference's full stage on the first n columns: depthkernelTI
    (surfdisp96 + tregn96 + splice) and depthkernel (1 + 6 nz surfdisp96)."""
    sl = lambda a: None if a is None else a[:n]  # noqa: E731
    O.depthkernel_ti(flat[:n], case.depz, case.periods, case.minthk, vp=sl(vp), rho=sl(rho),
                     nthreads=cores)
    O.depthkernel(flat[:n], case.depz, case.periods, case.minthk, vp=sl(vp), rho=sl(rho),
                  nthreads=cores)


def cpu_baseline(case, sample_s, form_kernels=True):
    """Oracle of the reference stage (depthkernelTI + depthkernel FD, the
    reference algorithm restated in C) on as many columns as fit in about
    sample_s seconds on all host threads; returns column-periods/s."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    flat = np.asfortranarray(case.vel.reshape(nx * ny, 1, nz))
    vp = None if case.vp is None else np.asfortranarray(case.vp.reshape(nx * ny, 1, nz))
    rho = None if case.rho is None else np.asfortranarray(case.rho.reshape(nx * ny, 1, nz))
    ncols = max(1, min(nx * ny, cores))
    t0 = time.perf_counter()
    _cpu_stage(O, flat, vp, rho, case, ncols, cores)
    t1 = time.perf_counter()
    per_col = (t1 - t0) / ncols * cores
    n2 = int(max(ncols, min(nx * ny, sample_s / max(per_col, 1e-9) * cores)))
    n2 = max(cores, (n2 // cores) * cores) if n2 >= cores else n2
    n2 = min(n2, nx * ny)
    t0 = time.perf_counter()
    _cpu_stage(O, flat, vp, rho, case, n2, cores)
    dt = time.perf_counter() - t0
    return {"value": n2 * K / dt, "unit": "column-periods/s", "cores": cores,
            "kind": "port",
            "sample": f"{n2} of {nx*ny} columns x {K} periods, oracle of depthkernelTI + "
                      f"depthkernel (FD: 1+6nz surfdisp96 per column), {dt:.1f} s on "
                      f"{cores} threads"}


def run_reference_ragged(args, ws, rank):
    """The reference's CPU path (the oracle restatement: the Fortran cannot
    be built here) on the host cores: each step times a fresh seeded sample
    of --cpu-cols-per-thread columns per thread drawn from the whole batch
    (8 by default: about 10 s of work on 16 threads); warm-up steps run one
    column per thread.  ms_per_step is the measured time of one sampled
    step."""
    if rank != 0:
        return
    from oracle import oracle as O
    b = load_ragged(args, 0)
    cores = os.cpu_count() or 1
    for w in range(args.warmup):
        sb = sub_batch(b, sample_columns(b, cores, 10_000 + w))
        O.batch(sb.node_off, sb.depz, sb.vs, sb.per_off, sb.periods, sb.minthk, nthreads=cores)
    vals, secs, cps = [], [], []
    for i in range(args.steps):
        cb, idx, sb, _ = ragged_cpu_baseline(b, seed=i, cores=cores,
                                             per_thread=args.cpu_cols_per_thread)
        vals.append(cb["value"])
        cps.append(sb.column_periods)
        secs.append(sb.column_periods / cb["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": "kernel column-periods/s", "value": v,
            "unit": "column-periods/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.median(secs)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": ragged_config(args, b),
            "cpu_baseline": {"value": v, "unit": "column-periods/s", "cores": cores,
                             "kind": "port",
                             "sample": f"median over {args.steps} steps; each step "
                                       f"{args.cpu_cols_per_thread * cores} seeded columns (seed = "
                                       f"step) of the {b.ncol}, {int(np.median(cps))} "
                                       f"column-periods (median), oracle of depthkernel (FD) "
                                       f"+ depthkernelTI at -O3 on {cores} threads"},
            "e2e": {"value": v, "unit": "column-periods/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ragged_config(args, b):
    nz = np.diff(b.node_off)
    K = np.diff(b.per_off)
    return {"workload": args.workload, "form": args.form, "columns": int(b.ncol),
            "column_periods": int(b.column_periods), "realisations": args.realisations,
            "layers_per_column": [int(nz.min()) - 1, int(nz.max()) - 1],
            "mean_layers": float(nz.mean() - 1), "periods_per_column": [int(K.min()), int(K.max())],
            "mean_periods": float(K.mean()), "minthk": b.minthk,
            "parallelism": "columns, one batch per GPU",
            "depth_cut": not getattr(args, "full_stack", False),
            "l2": "inputs and outputs far larger than L2; 256 MiB flush write between steps "
                  "outside the timed events"}


def _per_column_rel_l2(got, ref, off, K, nz, mask_k):
    """Worst per-column rel-L2 over the columns' (period, node) entries,
    periods k < mask_k[c] only (the periods with a root)."""
    worst = 0.0
    for c in range(K.size):
        kk = int(mask_k[c])
        if kk == 0:
            continue
        g = got[off[c]:off[c + 1]].reshape(nz[c], K[c])[:, :kk]
        r = ref[off[c]:off[c + 1]].reshape(nz[c], K[c])[:, :kk]
        den = np.linalg.norm(r)
        if den > 0:
            worst = max(worst, float(np.linalg.norm(g - r) / den))
    return worst


def accuracy_block(sb, gpu, ora, exact, plain):
    """Errors of the timed form on the sampled columns against the oracle:
    gpu / plain = the library's adjoint-form and plain-form outputs of those
    columns, ora = the oracle in the reference's arithmetic (FD kernels,
    Lsen_Gsc), exact = the oracle's exact-model differences (double model,
    roots to 1e-13, dln 1e-4)."""
    K = np.diff(sb.per_off)
    nz = np.diff(sb.node_off)
    sen_off = np.concatenate([[0], np.cumsum(K * nz)])
    ls_off = np.concatenate([[0], np.cumsum(K * (nz - 1))])
    pv_ref = ora["pv"]
    # status: first period without a root (1-based), 0 if none
    st_ref = np.zeros(K.size, np.int64)
    for c in range(K.size):
        z = np.nonzero(pv_ref[sb.per_off[c]:sb.per_off[c + 1]] == 0)[0]
        st_ref[c] = z[0] + 1 if z.size else 0
    good = np.where(st_ref > 0, st_ref - 1, K)
    ok = pv_ref > 0
    rel = np.abs(gpu["pv"][ok] / pv_ref[ok] - 1.0)
    same_status = gpu["status"] == st_ref
    within = np.zeros(pv_ref.size, bool)
    within[ok] = rel <= 1e-6
    ident = int(sum(bool(same_status[c]) and bool(within[sb.per_off[c]:sb.per_off[c] + good[c]].all())
                    for c in range(K.size)))
    ls_worst = 0.0
    for c in range(K.size):
        kk = int(good[c])
        if kk == 0:
            continue
        g = gpu["lsen"][ls_off[c]:ls_off[c + 1]].reshape(nz[c] - 1, K[c])[:, :kk]
        r = ora["lsen"][ls_off[c]:ls_off[c + 1]].reshape(nz[c] - 1, K[c])[:, :kk]
        den = np.linalg.norm(r.astype(np.float64))
        if den > 0:
            ls_worst = max(ls_worst, float(np.linalg.norm((g - r).astype(np.float64)) / den))
    names = ("sen_vs", "sen_vp", "sen_rho")
    ex_ok = ok & (exact["pv"] > 0)
    acc = {
        "columns": int(K.size), "column_periods": int(sb.column_periods),
        "pv_max_rel_err": float(rel.max()) if rel.size else 0.0,
        "pv_max_rel_err_vs_exact_root": float(np.abs(gpu["pv"][ex_ok] / exact["pv"][ex_ok] - 1.0).max())
        if ex_ok.any() else 0.0,
        "pv_bit_identical": int(np.count_nonzero(gpu["pv"] == pv_ref)),
        "status_equal_columns": int(same_status.sum()),
        "fundamental_mode_identity_columns": ident,
        "adjoint_kernels_vs_exact_worst_column_rel_l2":
            {n: _per_column_rel_l2(gpu[n], exact[n], sen_off, K, nz, good) for n in names},
        "adjoint_kernels_vs_reference_fd_worst_column_rel_l2":
            {n: _per_column_rel_l2(gpu[n], ora[n], sen_off, K, nz, good) for n in names},
        "lsen_worst_column_rel_l2": ls_worst,
        "tolerances": {"pv": 1e-6, "kernels_vs_exact": 1e-4,
                       "kernels_vs_reference_fd_gate": {"sen_vs": 1e-3, "sen_vp": 2e-3,
                                                        "sen_rho": 2e-3},
                       "lsen": 1e-5},
    }
    if plain is not None:
        acc["plain_form"] = {
            "pv_max_rel_err": float(np.abs(plain["pv"][ok] / pv_ref[ok] - 1.0).max()),
            "pv_bit_identical": int(np.count_nonzero(plain["pv"] == pv_ref)),
            "kernel_entries_bit_identical": int(sum(np.count_nonzero(plain[n] == ora[n])
                                                    for n in names)),
            "kernel_entries": int(3 * sen_off[-1]),
            "kernels_vs_reference_fd_worst_column_rel_l2":
                {n: _per_column_rel_l2(plain[n], ora[n], sen_off, K, nz, good) for n in names}}
    return acc


def run_reference(args, ws, rank):
    if args.workload == "config3":
        return run_reference_ragged(args, ws, rank)
    case = load_case(args.workload)
    if rank != 0:
        return
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    vals = []
    for _ in range(args.warmup):
        pass
    for _ in range(args.steps):
        cb = cpu_baseline(case, args.cpu_sample_s / max(args.steps, 1))
        vals.append(cb["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": "kernel column-periods/s", "value": v,
            "unit": "column-periods/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": nx * ny * K / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": args.workload, "columns": nx * ny,
                                            "periods": K, "nodes": nz, "minthk": case.minthk},
            "cpu_baseline": {"value": v, "unit": "column-periods/s", "cores": cb["cores"],
                             "kind": cb["kind"], "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "column-periods/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _events_timed(step, steps, warmup, dev, stream, flush, ws):
    """Per-step CUDA events on the launching stream; L2 flushed between steps
    outside the events; max over ranks.  Returns ms per step."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    for i in range(steps):
        flush.zero_()
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    total = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    if ws > 1:
        tt = torch.tensor([total], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        total = float(tt.item())
    return total / steps


def _work_constants():
    """FP64 operations and DRAM bytes per unit (root layer evaluation,
    adjoint and Gc/Gs layer item), counted by ncu (dadd + dmul + 2 dfma per
    thread instruction; dram__bytes_read + write) on captures of the uneven
    batch (the file names each) and divided by their units."""
    path = os.path.join(ROOT, "profiles", "kernel_work.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return {}


def main_ragged(args, ws, rank, local):
    import torch
    from dazi_current_release_b200 import _lib
    from dazi_current_release_b200.batch import output_offsets
    L = _lib.load(build_if_missing=False)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    b = load_ragged(args, rank)
    ncol = b.ncol
    sen_off, ls_off = output_offsets(b.node_off, b.per_off)
    form = _lib.FORM_PLAIN if args.form == "plain" else _lib.FORM_ADJOINT
    fast = form == _lib.FORM_ADJOINT and args.root == "brent"
    if fast:
        form |= _lib.FORM_FAST_ROOT
    if args.full_stack:
        form |= _lib.FORM_FULL_STACK
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    d_node, d_per, d_dep, d_vs = T(b.node_off), T(b.per_off), T(b.depz), T(b.vs)
    d_periods, d_senoff, d_lsoff = T(b.periods), T(sen_off), T(ls_off)
    ncp = int(b.per_off[-1])
    # whole-job column-periods: every rank has its own realisations
    job_cp = float(ncp)
    if ws > 1:
        tcp = torch.tensor([job_cp], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tcp, op=torch.distributed.ReduceOp.SUM)
        job_cp = float(tcp.item())
    pv = torch.zeros(ncp, dtype=torch.float64, device=dev)
    sen = [torch.zeros(int(sen_off[-1]), dtype=torch.float64, device=dev) for _ in range(3)]
    lsen = torch.zeros(int(ls_off[-1]), dtype=torch.float32, device=dev)
    status = torch.zeros(ncol, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    ptr = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731

    def step_fn(f, n):
        def step():
            rc = L.dazi_dk_batch_dev(n, ptr(d_node), ptr(d_dep), ptr(d_vs), None, None,
                                     ptr(d_per), ptr(d_periods), ctypes.c_float(b.minthk),
                                     ptr(pv), ptr(d_senoff), ptr(sen[0]), ptr(sen[1]),
                                     ptr(sen[2]), ptr(d_lsoff), ptr(lsen), f, ptr(status),
                                     ctypes.c_void_p(stream.cuda_stream))
            _lib.check(rc)
        return step

    def work():
        ev, lev, cpi, li = (ctypes.c_longlong(0) for _ in range(4))
        _lib.check(L.dazi_dk_last_work(ctypes.byref(ev), ctypes.byref(lev)))
        _lib.check(L.dazi_dk_last_items(ctypes.byref(cpi), ctypes.byref(li)))
        return ev.value, lev.value, li.value

    # both forms on the same sample of columns (the plain form on all 250k
    # columns would take minutes per step)
    ns = min(ncol, args.plain_cols)
    ns_cp = int(b.per_off[ns])
    sample = {}
    if not args.no_other_form:
        for fname, f in (("plain", _lib.FORM_PLAIN), ("adjoint", form)):
            ms = _events_timed(step_fn(f, ns), 1 if f == _lib.FORM_PLAIN else 2, 1, dev, stream,
                               flush, ws)
            sample[fname] = {"value": ws * ns_cp / (ms * 1e-3), "ms_per_step": ms}
    # per-call entry (tables rebuilt, one small host sync per call)
    call_ms = _events_timed(step_fn(form, ncol), max(2, args.steps // 2), 1, dev, stream, flush,
                            ws)
    launches_call = L.dazi_dk_last_launches()
    evals, layer_evals, layer_items = work()
    # plan: structure bound once, kernel variants autotuned on this batch,
    # every step one CUDA-graph launch (layer values from the current
    # velocities, root search, adjoint and Gc/Gs sweeps)
    graph_info = None
    if form & 1:
        from dazi_current_release_b200.plan import BatchPlan
        t0 = time.perf_counter()
        plan = BatchPlan(b.node_off, b.depz, b.vs, b.per_off, b.periods, b.minthk, tune=True,
                         scan32=bool(form & _lib.FORM_SCAN_FP32), fast_root=fast,
                         full_stack=args.full_stack, device=dev)
        plan_setup_s = time.perf_counter() - t0
        with ClockSampler(local) as clk:
            ms_per_step = _events_timed(plan.run, args.steps, args.warmup, dev, stream, flush, ws)
        plan.status_check()
        graph_info = {"autotuned": plan.config(), "setup_s": plan_setup_s,
                      "same_roots_as_per_call": bool(torch.equal(plan.pv, pv))
                      and bool(torch.equal(plan.status, status))}
        plan.close()
        launches = 6   # graph kernels per run: table values, root, adjoint order, adjoint,
        #                Gc/Gs order, Gc/Gs
    else:
        with ClockSampler(local) as clk:
            ms_per_step = _events_timed(step_fn(form, ncol), args.steps, args.warmup, dev,
                                        stream, flush, ws)
        launches = L.dazi_dk_last_launches()
    value = job_cp / (ms_per_step * 1e-3)

    # per-phase device times of one more step (events inside the library),
    # and of one step with every root-search evaluation in FP64
    _lib.check(L.dazi_dk_set_timing(1))
    torch.cuda.synchronize(dev)
    step_fn(form, ncol)()
    phases = _lib.last_timing()
    # outputs of the sampled columns (the CPU baseline's sample) for the
    # accuracy block, taken from this full-batch step
    acc_cols = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        acc_cols = sample_columns(b, args.cpu_cols_per_thread * (os.cpu_count() or 1), 0)
        gpu_sample = _gather_columns(torch, dev, b, acc_cols, sen_off, ls_off, pv, sen, lsen,
                                     status)
    scan32 = None
    root_search = None
    alt_sample = None
    alt_is_brent = False
    if form & _lib.FORM_ADJOINT:
        pv_t, st_t = pv.clone(), status.clone()
        sen_t = [x.clone() for x in sen]
        ls_t = lsen.clone()
        evals_t = evals
        # the other refinement of each period's bracket (the reference's
        # nevill() or Brent's, DAZI_FORM_FAST_ROOT), timed per call on the
        # same batch, and every output compared with the headline form's
        alt = form ^ _lib.FORM_FAST_ROOT
        _lib.check(L.dazi_dk_set_timing(0))
        alt_ms = _events_timed(step_fn(alt, ncol), max(2, args.steps // 2), 1, dev, stream, flush,
                               ws)
        _lib.check(L.dazi_dk_set_timing(1))
        step_fn(alt, ncol)()
        ph_alt = _lib.last_timing()
        ev_alt, lev_alt, _ = work()
        if acc_cols is not None:
            alt_sample = _gather_columns(torch, dev, b, acc_cols, sen_off, ls_off, pv, sen, lsen,
                                         status)
        ok = pv_t > 0
        rel = torch.where(ok, (pv / torch.where(ok, pv_t, 1.0) - 1.0).abs(), 0.0)
        grl = lambda a, r: float((torch.linalg.vector_norm(a - r) /  # noqa: E731
                                  torch.linalg.vector_norm(r)).item())
        brent = alt_is_brent = bool(alt & _lib.FORM_FAST_ROOT)
        ref_ph, brent_ph = (phases, ph_alt) if brent else (ph_alt, phases)
        root_search = {
            "refinement": "headline: " + ("reference nevill()" if brent else "Brent") +
                          "; other: " + ("Brent (DAZI_FORM_FAST_ROOT)" if brent else
                                         "reference nevill()") +
                          ".  Both run the reference's getsol scan point for point (same "
                          "bracket, same mode); Brent refines it to 1e-10 c, nevill() to 1e-6 c",
            "brent": {"value_per_call": job_cp / ((alt_ms if brent else call_ms) * 1e-3),
                      "root_ms": brent_ph.get("root"),
                      "evals_per_column_period": (ev_alt if brent else evals_t) / ncp},
            "reference": {"value_per_call": job_cp / ((call_ms if brent else alt_ms) * 1e-3),
                          "root_ms": ref_ph.get("root"),
                          "evals_per_column_period": (evals_t if brent else ev_alt) / ncp},
            "columns_same_status": int((st_t == status).sum().item()), "columns": ncol,
            "periods_same_root_presence": int(((pv > 0) == ok).sum().item()),
            "pv_max_rel_diff": float(rel.max().item()),
            "pv_within_reference_tolerance": int((rel <= 1e-6 + 1.3e-7).sum().item()),
            "column_periods": ncp,
            "kernels_rel_l2": {n: grl(sen[i], sen_t[i])
                               for i, n in enumerate(("sen_vs", "sen_vp", "sen_rho"))},
            "lsen_rel_l2": grl(lsen, ls_t),
            "note": "Lsen_Gsc follows the root: tregn96's partials at the reference's root "
                    "(converged to 1e-6 c) and at the exact root differ by up to 1 % per "
                    "period on sediment columns at short periods"}
        if not brent:
            layer_evals = lev_alt      # E_ref: the reference's evaluation sequence
        del sen_t, ls_t
        step_fn(form | _lib.FORM_SCAN_FP32, ncol)()
        ph32 = _lib.last_timing()
        scan32 = {"root_ms_fp64_scan": phases.get("root"), "root_ms_fp32_scan": ph32.get("root"),
                  "identical_roots": bool(torch.equal(pv_t, pv))}
    _lib.check(L.dazi_dk_set_timing(0))

    # end to end: host C-ABI dazi_dk_batch with pinned host buffers
    pin = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    h = {}
    for name, arr in (("node", b.node_off), ("per", b.per_off), ("dep", b.depz), ("vs", b.vs),
                      ("periods", b.periods), ("senoff", sen_off), ("lsoff", ls_off)):
        h[name] = pin(arr.size, {np.dtype(np.int64): torch.int64, np.dtype(np.float32): torch.float32,
                                 np.dtype(np.float64): torch.float64}[arr.dtype])
        h[name][:] = arr
    h_pv = pin(ncp, torch.float64)
    h_sen = [pin(int(sen_off[-1]), torch.float64) for _ in range(3)]
    h_ls = pin(int(ls_off[-1]), torch.float32)
    h_st = pin(ncol, torch.int32)
    CT = {np.dtype(np.int64): ctypes.c_longlong, np.dtype(np.float32): ctypes.c_float,
          np.dtype(np.float64): ctypes.c_double, np.dtype(np.int32): ctypes.c_int}

    def P(a):
        return a.ctypes.data_as(ctypes.POINTER(CT[a.dtype]))

    def e2e_step():
        rc = L.dazi_dk_batch(ncol, P(h["node"]), P(h["dep"]), P(h["vs"]), None, None,
                             P(h["per"]), P(h["periods"]), ctypes.c_float(b.minthk), P(h_pv),
                             P(h["senoff"]), P(h_sen[0]), P(h_sen[1]), P(h_sen[2]),
                             P(h["lsoff"]), P(h_ls), form, P(h_st))
        _lib.check(rc)

    e2e_step()
    e2e_steps = max(1, min(args.steps, 3))
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if ws > 1:
        tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(tt.item())
    h2d = sum(h[k].nbytes for k in h)
    d2h = h_pv.nbytes + sum(x.nbytes for x in h_sen) + h_ls.nbytes + h_st.nbytes

    # roofline of the dominant kernel.  achieved = algorithmic FP64 flops
    # (the hand count of 180 per layer of one secular evaluation) / the
    # kernel's event-timed duration: root search 180 x sum over column-periods
    # of rmax x E_ref (E_ref = the reference's evaluation count, which the
    # device search reproduces point for point); adjoint and Gc/Gs sweeps
    # 180 x 2 x layer items each (two forward-equivalent sweeps, the + 4 of
    # the whole-step count split between them).  pipe_frac: the FP64
    # operations ncu counts as executed (exp/sqrt/division included).
    peak = ctypes.c_double(0.0)
    _lib.check(L.dazi_dk_fp64_peak(ctypes.byref(peak)))
    peak_tf = peak.value / 1e3
    consts = _work_constants()
    units = {"root": ("layer_eval", layer_evals), "adjoint": ("layer_item", layer_items),
             "ti": ("layer_item", layer_items)}
    alg_flops = {"root": FLOP_PER_LAYER_EVAL * layer_evals,
                 "adjoint": FLOP_PER_LAYER_EVAL * SWEEP_FWD_EQUIV * layer_items,
                 "ti": FLOP_PER_LAYER_EVAL * SWEEP_FWD_EQUIV * layer_items}
    exec_flops, traffic_of = {}, {}
    for k, (uname, n) in units.items():
        f = consts.get(f"{k}_fp64_ops_per_{uname}")
        if f:
            exec_flops[k] = f * n
        t = consts.get(f"{k}_dram_bytes_per_{uname}")
        if t:
            traffic_of[k] = t * n
    ph = dict(phases)
    dom = max((n for n in ph if n != "prep"), key=lambda n: ph[n])
    tf = lambda fl, k: fl / (ph[k] * 1e-3) / 1e12  # noqa: E731
    achieved = tf(alg_flops[dom], dom) if dom in alg_flops else None
    traffic = traffic_of.get(dom)
    roof = {"bound": "fp64", "kernel": {"root": "root_kernel", "adjoint": "adjoint_kernel",
                                         "ti": "ti_kernel", "fd": "fd_batch_kernel"}.get(dom, dom),
            "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": achieved / peak_tf if achieved and peak_tf > 0 else None,
            "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per unit on a "
                              "capture of this workload (profiles/kernel_work.json), scaled by "
                              "the units of this launch",
            "peak_source": "measured in-run FP64 FMA probe (dazi_dk_fp64_peak); "
                           "MEASURED_PEAKS.json holds no FP64 figure",
            "kernel_ms": ph[dom], "flops_per_launch": alg_flops.get(dom),
            "formula": {"root": "180 x root_layer_evals_ref", "adjoint": "180 x 2 x layer_items",
                        "ti": "180 x 2 x layer_items", "frac": "flops_per_launch / kernel_ms / peak"},
            "flop_per_layer_eval": FLOP_PER_LAYER_EVAL,
            "phase_tflops": {k: tf(alg_flops[k], k) for k in alg_flops if k in ph},
            "phase_frac": {k: tf(alg_flops[k], k) / peak_tf for k in alg_flops if k in ph},
            "pipe_frac": {k: tf(exec_flops[k], k) / peak_tf for k in exec_flops if k in ph},
            "phase_ms": ph, "layer_items": layer_items, "secular_evals": evals,
            "root_layer_evals_ref": layer_evals}
    # algorithmic work of the whole step: sum over column-periods of
    # rmax x 180 x (E + 4), E = the root search's secular evaluations (the
    # reference's sequence of points), 180 FP64 flops per layer of one
    # evaluation (sqrt and division counted as one, transcendentals not
    # counted), + 4 forward-equivalent sweeps for the adjoint and Gc/Gs
    # kernels; sum rmax x E = root_layer_evals, sum rmax = layer_items
    alg = FLOP_PER_LAYER_EVAL * (layer_evals + 4 * layer_items)
    roof["algorithmic"] = {
        "flop_per_step": alg, "tflops": alg / (ms_per_step * 1e-3) / 1e12,
        "frac": alg / (ms_per_step * 1e-3) / 1e12 / peak_tf if peak_tf > 0 else None,
        "formula": "sum over column-periods of rmax x 180 x (E_ref + 4), over the whole step"}
    line = {
        "metric": "kernel column-periods/s", "value": value, "unit": "column-periods/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": dict(ragged_config(args, b),
                       root_refinement="brent" if fast else "reference nevill()"),
        "e2e": {"value": job_cp / e2e_s, "unit": "column-periods/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "roofline": roof,
        "gpu_launches": args.steps * launches,
        "graph": graph_info,
        "per_call": {"value": job_cp / (call_ms * 1e-3), "ms_per_step": call_ms,
                     "launches_per_call": launches_call},
    }
    if scan32:
        line["root_scan"] = scan32
    if root_search:
        line["root_search"] = root_search
    if sample:
        line["same_columns"] = dict(sample, columns=ns, column_periods=ns_cp,
                                    adjoint_over_plain=sample["adjoint"]["value"] /
                                    sample["plain"]["value"])
    clocks = clk.summary()
    if clocks:
        line["clocks"] = clocks
    if ws > 1:
        line["gather"] = _timed_gather(torch, dev, stream, pv, status, sen, lsen)
    if acc_cols is not None:
        from oracle import oracle as O
        cb, idx, sb, ora = ragged_cpu_baseline(b, seed=0, per_thread=args.cpu_cols_per_thread)
        assert np.array_equal(idx, acc_cols)
        line["cpu_baseline"] = cb
        t0 = time.perf_counter()
        exact = O.batch_fd(sb.node_off, sb.depz, sb.vs, sb.per_off, sb.periods, sb.minthk,
                           exact=True)
        plain = _run_sub_batch(torch, dev, L, _lib, sb, _lib.FORM_PLAIN)
        acc = accuracy_block(sb, gpu_sample, ora, exact, plain)
        acc["sample"] = (f"the cpu_baseline's {sb.ncol} columns; the adjoint form's outputs from "
                         f"the full-batch step, the plain form run on those columns alone; "
                         f"exact differences {time.perf_counter() - t0:.1f} s")
        if alt_sample is not None:
            brent_s = alt_sample if alt_is_brent else gpu_sample
            a2 = accuracy_block(sb, brent_s, ora, exact, None)
            args_sb = (sb.node_off, sb.depz, sb.vs, sb.per_off, sb.periods, sb.minthk)
            at_pv = O.batch_ti(*args_sb, pv=brent_s["pv"])
            tight = O.batch_ti(*args_sb, root_tol=1e-13)
            K = np.diff(sb.per_off)
            good = np.array([int(np.argmin(ora["pv"][sb.per_off[c]:sb.per_off[c + 1]] > 0))
                             if (ora["pv"][sb.per_off[c]:sb.per_off[c + 1]] <= 0).any() else K[c]
                             for c in range(sb.ncol)])
            lsen_w = lambda ref: max(  # noqa: E731
                (float(np.linalg.norm((brent_s["lsen"][a:e] - ref[a:e]).astype(np.float64)) /
                       np.linalg.norm(ref[a:e].astype(np.float64)))
                 for a, e in zip(at_pv["ls_off"][:-1], at_pv["ls_off"][1:])
                 if e > a and np.linalg.norm(ref[a:e]) > 0), default=0.0)
            tk = tight["pv"] > 0
            acc["brent_root"] = {
                "pv_max_rel_err": a2["pv_max_rel_err"],
                "pv_max_rel_err_vs_tight_root": float(np.abs(brent_s["pv"][tk] / tight["pv"][tk]
                                                              - 1.0).max()),
                "status_equal_columns": a2["status_equal_columns"],
                "fundamental_mode_identity_columns": a2["fundamental_mode_identity_columns"],
                "adjoint_kernels_vs_exact_worst_column_rel_l2":
                    a2["adjoint_kernels_vs_exact_worst_column_rel_l2"],
                "lsen_vs_oracle_at_same_pv_worst_column_rel_l2": lsen_w(at_pv["lsen"]),
                "lsen_vs_oracle_at_tight_root_worst_column_rel_l2": lsen_w(tight["lsen"]),
                "lsen_vs_oracle_reference_root_worst_column_rel_l2": a2["lsen_worst_column_rel_l2"],
                "tight_root": "surfdisp96 on the real*4 model converged to 1e-13, rounded to "
                              "float32", "periods_with_root": int(good.sum())}
        line["accuracy"] = acc
    if rank == 0 and ws == 1 and not args.no_fmm:
        line["fmm"] = fmm_block(torch, dev, stream, not args.no_cpu_baseline)
    if rank == 0 and ws == 1 and not args.no_lsmr:
        line["lsmr"] = lsmr_block(torch, dev, stream, not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def fmm_block(torch, dev, stream, with_cpu):
    """The traveltime solver on the Yunnan example's data set (1,469
    (period, source) fields, 20,877 receivers; tests/golden/yunnan_fmm.npz)
    through the initial model's phase-velocity maps (the library's
    surfdisp96 on tests/golden/yunnan_pv.npz's MOD, all 38 x 42 columns, 36
    periods): device-resident time (CUDA events, 3 runs after 2 warm-up),
    the host entry end to end (maps and coordinates copied in, times out),
    and the oracle on all host threads on the same input, whose times the
    GPU's must equal bit for bit."""
    import dazi_current_release_b200 as dk
    from dazi_current_release_b200 import fmm
    g = np.load(os.path.join(ROOT, "tests", "golden", "yunnan_fmm.npz"))
    m = np.load(os.path.join(ROOT, "tests", "golden", "yunnan_pv.npz"))
    vel, depz, per = m["vel"], m["depz"], m["periods"]
    nx, ny, nz = vel.shape
    pv = np.asfortranarray(dk.depthkernel(nx, ny, nz, vel, 2, 0, per.size, per, depz,
                                          float(m["minthk"]), form=dk.FORM_PLAIN,
                                          kernels=False)[0], np.float64).reshape(nx * ny, per.size,
                                                                                  order="F")
    st = g["station"][g["rc_station"]]
    inst = g["src_period"].astype(np.int32) - 1
    scx, scz = fmm.colatitude(g["src_lat"]), fmm.longitude(g["src_lon"])
    rcx, rcz = fmm.colatitude(st[:, 0]), fmm.longitude(st[:, 1])
    off = g["rc_off"].astype(np.int64)
    goxd, gozd, dvxd, dvzd = (float(v) for v in g["grid"])
    P = fmm.params(nx, ny, goxd, gozd, dvxd, dvzd)
    host_args = (pv, inst, scx, scz, off, rcx, rcz)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    dargs = (t(pv.T.copy().ravel()), t(inst), t(scx), t(scz), t(off), t(rcx), t(rcz))
    with torch.cuda.stream(stream):
        for _ in range(2):
            fmm.travel_times_dev(P, *dargs, stream=stream)
        stream.synchronize()
        ms = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fmm.travel_times_dev(P, *dargs, stream=stream)
            e1.record(stream)
            stream.synchronize()
            ms.append(e0.elapsed_time(e1))
    e2e = []
    for _ in range(3):
        t0 = time.perf_counter()
        times = fmm.travel_times(P, *host_args)
        e2e.append((time.perf_counter() - t0) * 1e3)
    assert np.array_equal(times, out.cpu().numpy())
    ninst, nrc = int(inst.size), int(off[-1])
    nnx, nnz = fmm.field_shape(P)
    dev_ms = float(np.median(ms))
    blk = {"workload": "Yunnan example data set: 1469 (period, source) traveltime fields on the "
                       f"{nnx} x {nnz} propagation grid with 129 x 129 refined source grids, "
                       f"{nrc} receiver times, initial-model phase-velocity maps",
           "instances": ninst, "receivers": nrc,
           "value": ninst / (dev_ms * 1e-3), "unit": "fields/s", "ms": dev_ms, "ms_runs": ms,
           "e2e": {"value": ninst / (float(np.median(e2e)) * 1e-3), "unit": "fields/s",
                   "ms": float(np.median(e2e)),
                   "h2d_bytes": int(pv.nbytes + 8 * ninst + 8 * (ninst + 1) + 8 * nrc),
                   "d2h_bytes": int(4 * nrc)},
           "bound": "latency: each field is one sequential narrow-band march (the reference's "
                    "heap order), one warp per field, all fields at once",
           "ns_per_node": dev_ms * 1e6 / (nnx * nnz + 129 * 129)}
    if with_cpu:
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        PO = O.fmm_params(nx, ny, goxd, gozd, dvxd, dvzd)
        t0 = time.perf_counter()
        ref = O.fmm_batch(PO, *host_args, nthreads=cores)
        cpu_s = time.perf_counter() - t0
        blk["cpu_baseline"] = {"value": ninst / cpu_s, "unit": "fields/s", "cores": cores,
                               "kind": "port", "sample": "the whole data set, oracle of "
                               "CalSurfG_parallel's per-(period, source) loop, one field per "
                               "thread at a time", "ms": cpu_s * 1e3}
        blk["times_equal_oracle"] = int(np.count_nonzero(times == ref))
    return blk


HBM_FALLBACK_GBS = 6650.0    # copy bandwidth of this pool's B200s, used when no measured file exists


def _hbm_peak():
    """(GB/s, source): MEASURED_PEAKS.json's copy bandwidth, else the
    fallback figure."""
    try:
        v = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
        return v, "measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError, KeyError, TypeError):
        return HBM_FALLBACK_GBS, "fallback 6.65 TB/s copy bandwidth (no measured file)"


def lsmr_block(torch, dev, stream, with_cpu):
    """The LSMR solver (dazi_lsmr_dev / dazi_lsmr) on a seeded G-like system
    with the Yunnan example's shape: 20,877 ray rows over the 38 x 42 cells,
    17 depth layers each (synthetic.g_like_system), plus one smoothing row
    per parameter; all tolerances 0, so every run takes exactly its
    iteration count.  Device-resident time with CUDA events (the call
    includes the CSR build); the marginal time per iteration from runs of
    ITERS and ITERS / 4 iterations, against the HBM roofline of its
    algorithmic bytes (both CSR copies, 8 B per non-zero each, the row
    pointers and the dense vectors); the host entry end to end; SciPy's
    lsmr (the reference's SciPy backend, oracle/lsmr_ref.py) on one host
    thread for CPU_ITERS iterations; and the first 10 iterations against
    SciPy's."""
    from dazi_current_release_b200 import _lib
    from dazi_current_release_b200.lsmr import lsmr
    from dazi_current_release_b200.synthetic import g_like_system
    ITERS, CPU_ITERS = 400, 100
    row, col, val, b, m, n = g_like_system(nvx=38, nvz=42, nz=17, nrays=20877, seed=0)
    nnz = int(val.size)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    drow, dcol, dval, db = t(row), t(col), t(val), t(b)
    kw = dict(atol=0.0, btol=0.0, conlim=0.0)

    def run(iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = lsmr(drow, dcol, dval, db, m, n, maxiter=iters, stream=stream.cuda_stream, **kw)
        e1.record(stream)
        stream.synchronize()
        assert (r.istop, r.itn) == (7, iters)
        return e0.elapsed_time(e1), r

    with torch.cuda.stream(stream):
        for _ in range(2):
            run(ITERS)
        full = [run(ITERS)[0] for _ in range(5)]
        part = [run(ITERS // 4)[0] for _ in range(5)]
        _, r10 = run(10)
        _, rk = run(ITERS)
    ms_full, ms_part = float(np.median(full)), float(np.median(part))
    it_ms = (ms_full - ms_part) / (ITERS - ITERS // 4)
    # the host waits once per 16 iterations, so a busy host shows in the
    # device time too: the least-disturbed runs beside the medians
    it_ms_best = (min(full) - min(part)) / (ITERS - ITERS // 4)
    # algorithmic bytes of one iteration: A v and A^T u (values 4 B + column
    # 4 B per non-zero, 8 B row pointers, the result read and written, the
    # gathered vector once), the vector update (h, h-bar, x, v read; h,
    # h-bar, x written)
    it_bytes = 2 * 8 * nnz + 8 * (m + 1) + 8 * (n + 1) + 8 * (3 * m + n) + 8 * (3 * n + m) + 8 * 7 * n
    peak, peak_src = _hbm_peak()
    # host entry: the Fortran-shaped call (iw = rows then columns, rw,
    # b in, x out), wall clock
    L = _lib.load()
    iw = np.concatenate([row, col]).astype(np.int32)
    ci, cl, cd = ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    P = lambda a, ty: a.ctypes.data_as(ctypes.POINTER(ty))  # noqa: E731
    xh = np.zeros(n, np.float64)
    e2e = []
    for _ in range(3):
        istop, itn = ci(0), ci(0)
        outs = [cd(0.0) for _ in range(5)]
        t0 = time.perf_counter()
        rc = L.dazi_lsmr(ctypes.byref(ci(m)), ctypes.byref(ci(n)), ctypes.byref(cl(iw.size)),
                         ctypes.byref(cl(nnz)), P(iw, ci), P(val, ctypes.c_float), P(b, cd),
                         ctypes.byref(cd(0.0)), ctypes.byref(cd(0.0)), ctypes.byref(cd(0.0)),
                         ctypes.byref(cd(0.0)), ctypes.byref(ci(ITERS)), ctypes.byref(ci(0)),
                         ctypes.byref(ci(6)), P(xh, cd), ctypes.byref(istop), ctypes.byref(itn),
                         *[ctypes.byref(o) for o in outs])
        e2e.append((time.perf_counter() - t0) * 1e3)
        _lib.check(rc)
    assert np.array_equal(xh, rk.x.cpu().numpy())
    e2e_ms = float(np.median(e2e))
    blk = {"workload": f"G-like system with the Yunnan example's shape: {m} x {n} ({20877} ray "
                       f"rows over 38 x 42 cells x 17 layers, plus {n} smoothing rows), "
                       f"{nnz} non-zeros, real*4 values, all tolerances 0",
           "m": m, "n": n, "nnz": nnz,
           "value": ITERS / (ms_full * 1e-3), "unit": "iterations/s",
           "solve_ms": ms_full, "iterations": ITERS, "solve_ms_runs": full,
           "ms_per_iteration": it_ms, "ms_per_iteration_best_runs": it_ms_best,
           "part_ms_runs": part,
           "e2e": {"value": ITERS / (e2e_ms * 1e-3), "unit": "iterations/s", "ms": e2e_ms,
                   "h2d_bytes": int(iw.nbytes + val.nbytes + b.nbytes), "d2h_bytes": int(8 * n)},
           "roofline": {"bound": "hbm", "achieved": it_bytes / (it_ms_best * 1e-3) / 1e9,
                        "peak": peak, "unit": "GB/s",
                        "frac": it_bytes / (it_ms_best * 1e-3) / 1e9 / peak,
                        "time": "ms_per_iteration_best_runs (each call also allocates its "
                                "buffers and builds its CSR copies on the host's schedule, so "
                                "busy hosts spread the medians)",
                        "bytes_per_iteration": it_bytes, "peak_source": peak_src,
                        "note": "marginal time per iteration, (t(ITERS) - t(ITERS/4)) / "
                                "(3 ITERS / 4), 6 launches per iteration in 16-iteration CUDA "
                                "graphs; the two CSR copies (143 MB) are about L2's size. The "
                                "products are bound by load latency, not by HBM: each warp "
                                "walks its rows one after another (rounds of column and value "
                                "loads, then their gathers), over uneven rows"}}
    if with_cpu:
        from oracle import lsmr_ref
        t0 = time.perf_counter()
        ref = lsmr_ref.lsmr(row, col, val, b, m, n, maxiter=CPU_ITERS, **kw)
        cpu_s = time.perf_counter() - t0
        ref10 = lsmr_ref.lsmr(row, col, val, b, m, n, maxiter=10, **kw)
        x10 = r10.x.cpu().numpy()
        blk["cpu_baseline"] = {"value": CPU_ITERS / cpu_s, "unit": "iterations/s", "cores": 1,
                               "kind": "port", "sample": f"{CPU_ITERS} iterations of SciPy's lsmr "
                               "on the same triplets (coo -> csr, float64), as the reference's "
                               "SciPy backend runs it; SciPy's sparse products use one thread",
                               "ms": cpu_s * 1e3, "itn": int(ref[2])}
        blk["x_rel_diff_vs_scipy_10_iterations"] = float(
            np.linalg.norm(x10 - ref10[0]) / np.linalg.norm(ref10[0]))
    return blk


def _timed_gather(torch, dev, stream, pv, status, sen, lsen):
    """The stage's one communication step: every rank's outputs (pv,
    status, the three kernels, Lsen_Gsc) gathered to rank 0 in rank order
    (shard.gather_blocks: size exchange, NCCL point-to-point receives into
    slices of rank 0's arrays).  Device time with CUDA events, max over
    ranks; the bytes rank 0 receives from the others."""
    import torch.distributed as dist
    from dazi_current_release_b200.shard import gather_blocks
    blocks = {"pv": pv, "status": status, "sen_vs": sen[0], "sen_vp": sen[1],
              "sen_rho": sen[2], "lsen": lsen}
    own = sum(t.numel() * t.element_size() for t in blocks.values())
    gather_blocks({"pv": pv[:1]})          # warm-up (NCCL communicators)
    torch.cuda.synchronize(dev)
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = gather_blocks(blocks)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    tot = torch.tensor([own], dtype=torch.float64, device=dev)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    received = float(tot.item()) - own if dist.get_rank() == 0 else None
    del out
    res = {"ms": float(ms.item()), "bytes_to_rank0": received,
           "what": "pv, status, sen_vs/vp/rho, Lsen_Gsc of every rank to rank 0 (NCCL "
                   "point-to-point into slices of preallocated arrays)"}
    if received:
        res["GB_per_s"] = received / (res["ms"] * 1e-3) / 1e9
    return res


def _gather_columns(torch, dev, b, idx, sen_off, ls_off, pv, sen, lsen, status):
    """Host copies of the outputs of columns idx (batch layout, in order)."""
    rng = lambda off: np.concatenate([np.arange(off[c], off[c + 1]) for c in idx])  # noqa: E731
    take = lambda t, i: t.index_select(0, torch.from_numpy(i).to(dev)).cpu().numpy()  # noqa: E731
    ip, isn, il = rng(b.per_off), rng(sen_off), rng(ls_off)
    return {"pv": take(pv, ip), "sen_vs": take(sen[0], isn), "sen_vp": take(sen[1], isn),
            "sen_rho": take(sen[2], isn), "lsen": take(lsen, il),
            "status": take(status, idx.astype(np.int64))}


def _run_sub_batch(torch, dev, L, _lib, sb, form):
    """One dazi_dk_batch_dev call on a small batch; host copies of its
    outputs (kernels, no Lsen_Gsc)."""
    from dazi_current_release_b200.batch import output_offsets
    sen_off, _ = output_offsets(sb.node_off, sb.per_off)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    d = [T(sb.node_off), T(sb.depz), T(sb.vs), T(sb.per_off), T(sb.periods), T(sen_off)]
    pv = torch.zeros(sb.column_periods, dtype=torch.float64, device=dev)
    sen = [torch.zeros(int(sen_off[-1]), dtype=torch.float64, device=dev) for _ in range(3)]
    st = torch.zeros(sb.ncol, dtype=torch.int32, device=dev)
    P = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    _lib.check(L.dazi_dk_batch_dev(sb.ncol, P(d[0]), P(d[1]), P(d[2]), None, None, P(d[3]),
                                   P(d[4]), ctypes.c_float(sb.minthk), P(pv), P(d[5]),
                                   P(sen[0]), P(sen[1]), P(sen[2]), None, None, form, P(st),
                                   ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    torch.cuda.synchronize(dev)
    return {"pv": pv.cpu().numpy(), "sen_vs": sen[0].cpu().numpy(),
            "sen_vp": sen[1].cpu().numpy(), "sen_rho": sen[2].cpu().numpy(),
            "status": st.cpu().numpy()}


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.workload == "config3":
        main_ragged(args, ws, rank, local)
        return
    import torch
    from dazi_current_release_b200 import _lib
    from dazi_current_release_b200.depthkernel import _run_fused
    L = _lib.load(build_if_missing=False)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    case = load_case(args.workload)
    nx, ny, nz = case.vel.shape
    K = case.periods.size
    nxy = nx * ny
    form = _lib.FORM_PLAIN if args.form == "plain" else _lib.FORM_ADJOINT

    # ---------------- device-resident timing (value)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dev)  # noqa: E731
    vel = t(case.vel)
    vp = None if case.vp is None else t(case.vp)
    rho = None if case.rho is None else t(case.rho)
    per = torch.from_numpy(case.periods.copy()).to(dev)
    depz = torch.from_numpy(case.depz.copy()).to(dev)
    pv = torch.zeros(nxy * K, dtype=torch.float64, device=dev)
    sen = [torch.zeros(nxy * K * nz, dtype=torch.float64, device=dev) for _ in range(3)]
    lsen = torch.zeros(nxy * K * (nz - 1), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    ptr = lambda x: None if x is None else ctypes.c_void_p(x.data_ptr())  # noqa: E731

    def step(f):
        rc = L.dazi_dk_fused_dev(nx, ny, nz, ptr(vel), ptr(vp), ptr(rho), ptr(pv), ptr(sen[0]),
                                 ptr(sen[1]), ptr(sen[2]), ptr(lsen), K, ptr(per), ptr(depz),
                                 ctypes.c_float(case.minthk), 1, nxy, f, None,
                                 ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc)

    def timed(f, steps, warmup, sampler=None):
        for _ in range(warmup):
            step(f)
        torch.cuda.synchronize(dev)
        ev = ctypes.c_longlong(0)
        lev = ctypes.c_longlong(0)
        _lib.check(L.dazi_dk_last_work(ctypes.byref(ev), ctypes.byref(lev)))
        launches = L.dazi_dk_last_launches()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
        for i in range(steps):
            flush.zero_()                      # L2 flush, outside the timed events
            starts[i].record(stream)
            step(f)
            ends[i].record(stream)
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        total = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
        if ws > 1:
            tt = torch.tensor([total], dtype=torch.float64, device=dev)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            total = float(tt.item())
        return total / steps, ev.value, lev.value, launches

    other = None
    if not args.no_other_form:
        of = _lib.FORM_PLAIN if form == _lib.FORM_ADJOINT else _lib.FORM_ADJOINT
        o_steps = max(1, min(args.steps, 2))
        oms, _, olev, _ = timed(of, o_steps, 1)
        other = {"form": "plain" if of == _lib.FORM_PLAIN else "adjoint",
                 "value": ws * nxy * K / (oms * 1e-3), "ms_per_step": oms, "steps": o_steps,
                 "flops_per_step": olev * FLOP_PER_LAYER_EVAL}
    with ClockSampler(local) as clk:
        ms_per_step, evals_per_step, layer_evals_per_step, launches = timed(
            form, args.steps, args.warmup)
    value = ws * nxy * K / (ms_per_step * 1e-3)

    # ---------------- end to end through the host C-ABI (pinned buffers)
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    h_vel = pin((nxy * nz,), torch.float32)
    h_vel[:] = case.vel.ravel(order="F")
    h_vel = h_vel.reshape((nx, ny, nz), order="F")
    h_pv = pin((nxy * K,), torch.float64).reshape((nxy, K), order="F")
    h_sen = tuple(pin((nxy * K * nz,), torch.float64).reshape((nxy, K, nz), order="F")
                  for _ in range(3))
    h_lsen = pin((nxy * K * (nz - 1),), torch.float32).reshape((nxy, K, nz - 1), order="F")
    if case.vp is not None:
        h_vp = pin((nxy * nz,), torch.float32)
        h_vp[:] = case.vp.ravel(order="F")
        h_rho = pin((nxy * nz,), torch.float32)
        h_rho[:] = case.rho.ravel(order="F")
        h_vp = h_vp.reshape((nx, ny, nz), order="F")
        h_rho = h_rho.reshape((nx, ny, nz), order="F")
    else:
        h_vp = h_rho = None

    def e2e_step():
        _run_fused(nx, ny, nz, h_vel, h_vp, h_rho, 2, 0, K, case.periods, case.depz, case.minthk,
                   form, 1, None, True, True, pvRc=h_pv, sen=h_sen, Lsen=h_lsen)

    e2e_step()
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if ws > 1:
        tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(tt.item())
    h2d = nxy * nz * 4 * (3 if case.vp is not None else 1) + K * 8
    d2h = nxy * K * 8 * (1 + 3 * nz) + nxy * K * 4 * (nz - 1) + nxy * 4

    # ---------------- roofline
    peak = ctypes.c_double(0.0)
    _lib.check(L.dazi_dk_fp64_peak(ctypes.byref(peak)))
    flops = layer_evals_per_step * _work_constants().get("root_fp64_ops_per_layer_eval",
                                                         FLOP_PER_LAYER_EVAL)
    achieved = flops / (ms_per_step * 1e-3) / 1e12
    peak_tf = peak.value / 1e3
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            tr = json.load(open(tpath))
            traffic = tr.get(f"{args.workload}:{args.form}")
        except (ValueError, OSError):
            traffic = None

    line = {
        "metric": "kernel column-periods/s", "value": value, "unit": "column-periods/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "form": args.form, "columns": nxy, "periods": K,
                   "nodes": nz, "minthk": case.minthk, "parallelism": f"columns x {ws} GPU",
                   "l2": "flushed between steps (256 MiB write outside the timed events)"},
        "e2e": {"value": ws * nxy * K / e2e_s, "unit": "column-periods/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": achieved / peak_tf if peak_tf > 0 else None, "traffic": traffic,
                     "peak_source": "measured in-run FP64 FMA probe (dazi_dk_fp64_peak)",
                     "flops_per_step": flops, "secular_evals_per_step": evals_per_step},
        "gpu_launches": args.steps * launches,
    }
    if other:
        line[other["form"]] = other
        line[args.form] = {"form": args.form, "value": value, "ms_per_step": ms_per_step}
    clocks = clk.summary()
    if clocks:
        line["clocks"] = clocks
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(case, args.cpu_sample_s)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
