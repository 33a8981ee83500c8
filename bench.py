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
           adjoint form) on the whole batch, inputs resident in HBM: a plan
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
           inside the library): root search 180 FP64 flops per layer per
           secular evaluation (evaluations counted by the kernel); adjoint and
           Gc/Gs sweeps the FP64 operations per layer item counted by ncu
           (profiles/kernel_work.json) x the layer items of the call; peak the
           FP64 FMA rate measured live by dazi_dk_fp64_peak
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

FLOP_PER_LAYER_EVAL = 180   # hand count of dltar4's FP64 arithmetic per layer (fallback when
                             # the ncu-counted figure is absent)


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
    p.add_argument("--no-other-form", action="store_true")
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-sample-s", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
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


def ragged_cpu_baseline(b, sample_s, cores=None):
    """Oracle of the reference stage (depthkernel FD + depthkernelTI per
    column, OpenMP over columns) on the first columns of the batch, as many
    as fit in about sample_s seconds; returns column-periods/s."""
    from oracle import oracle as O
    cores = cores or os.cpu_count() or 1

    def run(n):
        no, po = b.node_off[:n + 1], b.per_off[:n + 1]
        t0 = time.perf_counter()
        O.batch(no, b.depz[:no[-1]], b.vs[:no[-1]], po, b.periods[:po[-1]], b.minthk,
                nthreads=cores)
        return time.perf_counter() - t0

    n1 = min(b.ncol, cores)
    dt1 = run(n1)
    n2 = int(min(b.ncol, max(n1, sample_s / max(dt1, 1e-9) * n1)))
    dt = run(n2) if n2 > n1 else dt1
    cp = int(b.per_off[n2])
    return {"value": cp / dt, "unit": "column-periods/s", "cores": cores, "kind": "port",
            "sample": f"first {n2} of {b.ncol} columns ({cp} column-periods), oracle of "
                      f"depthkernel (FD: 1+6nz surfdisp96 per column) + depthkernelTI, "
                      f"{dt:.1f} s on {cores} threads"}


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
    if rank != 0:
        return
    b = load_ragged(args, 0)
    vals = []
    for _ in range(args.steps):
        cb = ragged_cpu_baseline(b, args.cpu_sample_s / max(args.steps, 1))
        vals.append(cb["value"])
    v = float(np.median(vals))
    cp = b.column_periods
    line = {"impl": "reference", "metric": "kernel column-periods/s", "value": v,
            "unit": "column-periods/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cp / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": ragged_config(args, b),
            "cpu_baseline": {"value": v, "unit": "column-periods/s", "cores": cb["cores"],
                             "kind": cb["kind"], "sample": cb["sample"]},
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
            "parallelism": "columns, one batch per GPU"}


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
    Gc/Gs layer item), counted by ncu (dadd + dmul + 2 dfma per thread
    instruction; dram__bytes_read + write) on a 100000-column capture of the
    uneven batch and divided by its units."""
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
        for fname, f in (("plain", _lib.FORM_PLAIN), ("adjoint", _lib.FORM_ADJOINT)):
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
                         scan32=bool(form & _lib.FORM_SCAN_FP32), device=dev)
        plan_setup_s = time.perf_counter() - t0
        with ClockSampler(local) as clk:
            ms_per_step = _events_timed(plan.run, args.steps, args.warmup, dev, stream, flush, ws)
        plan.status_check()
        graph_info = {"autotuned": plan.config(), "setup_s": plan_setup_s,
                      "same_roots_as_per_call": bool(torch.equal(plan.pv, pv))
                      and bool(torch.equal(plan.status, status))}
        plan.close()
        launches = 4   # graph kernels per run: table values, root, adjoint, Gc/Gs
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
    scan32 = None
    if form == _lib.FORM_ADJOINT:
        pv64 = pv.clone()
        step_fn(form | _lib.FORM_SCAN_FP32, ncol)()
        ph32 = _lib.last_timing()
        scan32 = {"root_ms_fp64_scan": phases.get("root"), "root_ms_fp32_scan": ph32.get("root"),
                  "identical_roots": bool(torch.equal(pv64, pv))}
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

    # roofline of the dominant kernel
    peak = ctypes.c_double(0.0)
    _lib.check(L.dazi_dk_fp64_peak(ctypes.byref(peak)))
    peak_tf = peak.value / 1e3
    consts = _work_constants()
    units = {"root": ("layer_eval", layer_evals), "adjoint": ("layer_item", layer_items),
             "ti": ("layer_item", layer_items)}
    flops, traffic_of = {}, {}
    for k, (uname, n) in units.items():
        f = consts.get(f"{k}_fp64_ops_per_{uname}")
        if f is None and k == "root":
            f = FLOP_PER_LAYER_EVAL
        if f:
            flops[k] = f * n
        t = consts.get(f"{k}_dram_bytes_per_{uname}")
        if t:
            traffic_of[k] = t * n
    ph = dict(phases)
    dom = max((n for n in ph if n != "prep"), key=lambda n: ph[n])
    achieved = flops[dom] / (ph[dom] * 1e-3) / 1e12 if dom in flops else None
    traffic = traffic_of.get(dom)
    roof = {"bound": "fp64", "kernel": {"root": "root_kernel", "adjoint": "adjoint_kernel",
                                         "ti": "ti_kernel", "fd": "fd_batch_kernel"}.get(dom, dom),
            "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": achieved / peak_tf if achieved and peak_tf > 0 else None,
            "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per unit on a "
                              "100000-column capture of this workload (profiles/kernel_work.json), "
                              "scaled by the units of this launch",
            "phase_tflops": {k: flops[k] / (ph[k] * 1e-3) / 1e12 for k in flops if k in ph},
            "peak_source": "measured in-run FP64 FMA probe (dazi_dk_fp64_peak)",
            "kernel_ms": ph[dom], "flops_per_launch": flops.get(dom),
            "phase_ms": ph, "layer_items": layer_items, "secular_evals": evals,
            "root_layer_evals": layer_evals}
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
                       l2="inputs and outputs far larger than L2; 256 MiB flush write between "
                          "steps outside the timed events"),
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
    if sample:
        line["same_columns"] = dict(sample, columns=ns, column_periods=ns_cp,
                                    adjoint_over_plain=sample["adjoint"]["value"] /
                                    sample["plain"]["value"])
    clocks = clk.summary()
    if clocks:
        line["clocks"] = clocks
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = ragged_cpu_baseline(b, args.cpu_sample_s)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


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
