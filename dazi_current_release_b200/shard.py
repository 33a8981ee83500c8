"""Columns over several GPUs: one process per GPU, contiguous column shards,
no exchange during the computation and one gather of the outputs at the end.

Every (column, period) of the stage depends only on its own column (and on
the previous period's root of that column), so the stage splits into
independent column ranges, the `col_start`/`col_count` contract of the
reference's tile worker (code/depthkernel_lab/depthkernel_ti_worker.f90:19-38)
carried over to the ragged batch.  Shards are balanced by an estimate of the
work of each column (periods x refined layers, the unit of the adjoint and
Gc/Gs sweeps).  The outputs of the ranks are gathered to one rank in the
batch's own CSR layout.
"""
from __future__ import annotations

import numpy as np

from .batch import output_offsets


def column_work(node_off, per_off, minthk):
    """Work estimate per column: periods x (refined layers) with the
    sublayer rule of refineGrid2LayerMdl (minthk + 1 sublayers per layer,
    plus the half-space)."""
    nz = np.diff(np.asarray(node_off, np.int64))
    K = np.diff(np.asarray(per_off, np.int64))
    ns = int(minthk) + 1
    return K * ((nz - 1) * ns + 1)


def shard_bounds(work, world: int):
    """Contiguous shard boundaries [b_0 = 0, ..., b_world = ncols] with
    nearly equal cumulative work (every rank gets at least one column when
    there are enough columns)."""
    work = np.asarray(work, np.float64)
    n = work.size
    if world < 1:
        raise ValueError("world must be >= 1")
    cum = np.concatenate([[0.0], np.cumsum(work)])
    targets = cum[-1] * np.arange(1, world) / world
    inner = np.searchsorted(cum, targets, side="left")
    b = np.concatenate([[0], inner, [n]]).astype(np.int64)
    b = np.maximum.accumulate(np.clip(b, 0, n))
    return b


def slice_batch(node_off, depz, vs, per_off, periods, c0: int, c1: int, vp=None, rho=None):
    """Columns c0..c1-1 of a ragged batch with offsets re-based to 0."""
    node_off = np.asarray(node_off, np.int64)
    per_off = np.asarray(per_off, np.int64)
    a, b = node_off[c0], node_off[c1]
    p, q = per_off[c0], per_off[c1]
    out = dict(node_off=node_off[c0:c1 + 1] - a, depz=np.asarray(depz)[a:b],
               vs=np.asarray(vs)[a:b], per_off=per_off[c0:c1 + 1] - p,
               periods=np.asarray(periods)[p:q])
    if vp is not None:
        out["vp"] = np.asarray(vp)[a:b]
        out["rho"] = np.asarray(rho)[a:b]
    return out


def _default_compute(part, minthk, form):
    from .batch import depthkernel_batch
    kw = {k: part[k] for k in ("vp", "rho") if k in part}
    return depthkernel_batch(part["node_off"], part["depz"], part["vs"], part["per_off"],
                             part["periods"], minthk, form=form, **kw)


def run_sharded(node_off, depz, vs, per_off, periods, minthk, *, form=1, vp=None, rho=None,
                compute=None, group=None, dst: int = 0):
    """Run this rank's shard of a ragged batch and gather every rank's
    outputs to rank `dst` (torch.distributed, any backend).  Returns the
    whole batch's outputs on `dst` (keys pv, sen_vs, sen_vp, sen_rho,
    lsen, status, in dazi_dk_batch's layout) and this rank's own shard
    result elsewhere.  `compute(part, minthk, form)` runs one shard; the
    default is the GPU batch entry (dazi_dk_batch)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    node_off = np.asarray(node_off, np.int64)
    per_off = np.asarray(per_off, np.int64)
    bounds = shard_bounds(column_work(node_off, per_off, minthk), world)
    c0, c1 = int(bounds[rank]), int(bounds[rank + 1])
    part = slice_batch(node_off, depz, vs, per_off, periods, c0, c1, vp, rho)
    res = (compute or _default_compute)(part, minthk, form)
    mine = {k: (None if res.get(k) is None else np.asarray(res[k]))
            for k in ("pv", "sen_vs", "sen_vp", "sen_rho", "lsen", "status")}
    mine["range"] = (c0, c1)
    gathered = [None] * world if rank == dst else None
    dist.gather_object(mine, gathered, dst=dst, group=group)
    if rank != dst:
        return mine
    # reassemble in the whole batch's CSR layout
    sen_off, ls_off = output_offsets(node_off, per_off)
    ncol = node_off.size - 1
    out = {"pv": np.zeros(int(per_off[-1])), "status": np.zeros(ncol, np.int32),
           "per_off": per_off, "sen_off": sen_off, "ls_off": ls_off}
    have_sen = any(g["sen_vs"] is not None for g in gathered)
    have_ls = any(g["lsen"] is not None for g in gathered)
    if have_sen:
        for k in ("sen_vs", "sen_vp", "sen_rho"):
            out[k] = np.zeros(int(sen_off[-1]))
    if have_ls:
        out["lsen"] = np.zeros(int(ls_off[-1]), np.float32)
    for g in gathered:
        a, b = g["range"]
        if b <= a:
            continue
        out["pv"][per_off[a]:per_off[b]] = g["pv"]
        out["status"][a:b] = g["status"]
        if have_sen:
            for k in ("sen_vs", "sen_vp", "sen_rho"):
                out[k][sen_off[a]:sen_off[b]] = g[k]
        if have_ls:
            out["lsen"][ls_off[a]:ls_off[b]] = g["lsen"]
    return out
