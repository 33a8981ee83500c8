"""Columns over several GPUs: one process per GPU, contiguous column shards,
no exchange during the computation and one gather of the outputs at the end.

Every (column, period) of the stage depends only on its own column (and on
the previous period's root of that column), so the stage splits into
independent column ranges, the `col_start`/`col_count` contract of the
reference's tile worker (code/depthkernel_lab/depthkernel_ti_worker.f90:19-38)
carried over to the ragged batch.  Shards are balanced by an estimate of the
work of each column (periods x refined layers, the unit of the adjoint and
Gc/Gs sweeps).  The outputs of the ranks are gathered to one rank in the
batch's own CSR layout: since the shards are contiguous column ranges in
rank order, every output array of the whole batch is the concatenation of
the ranks' arrays, so the gather is one exchange of block sizes and
point-to-point receives of each rank's blocks straight into slices of the
destination's preallocated arrays (NCCL for device tensors, gloo for host
tensors; no pickling).
"""
from __future__ import annotations

import numpy as np

from .batch import output_offsets

OUTPUT_KEYS = ("pv", "status", "sen_vs", "sen_vp", "sen_rho", "lsen")


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


def gather_blocks(blocks, dst: int = 0, group=None):
    """Concatenate every rank's 1-D tensors key by key, in rank order, on
    rank `dst`.  blocks: {key: tensor or None}, the same keys with the same
    dtypes on every rank, all on one device (CUDA for NCCL, CPU for gloo).
    Returns {key: whole tensor} on dst and None elsewhere.  Every rank makes
    the same collective calls in the same order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    keys = [k for k in blocks if blocks[k] is not None]
    dev = blocks[keys[0]].device
    n = torch.tensor([blocks[k].numel() for k in keys], dtype=torch.int64, device=dev)
    sizes = [torch.empty_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = torch.stack(sizes).cpu().numpy()           # [rank, key]
    starts = np.concatenate([np.zeros((1, len(keys)), np.int64), np.cumsum(sizes, axis=0)])
    peer = (lambda r: dist.get_global_rank(group, r)) if group is not None else (lambda r: r)
    reqs, out = [], {}
    for j, k in enumerate(keys):
        t = blocks[k].contiguous()
        if rank == dst:
            full = torch.empty(int(starts[-1, j]), dtype=t.dtype, device=dev)
            full[starts[rank, j]:starts[rank + 1, j]].copy_(t)
            for r in range(world):
                a, b = int(starts[r, j]), int(starts[r + 1, j])
                if r != dst and b > a:
                    reqs.append(dist.irecv(full[a:b], src=peer(r), group=group))
            out[k] = full
        elif t.numel() > 0:
            reqs.append(dist.isend(t, dst=peer(dst), group=group))
    for q in reqs:
        q.wait()
    return out if rank == dst else None


def _default_compute(part, minthk, form):
    from .batch import depthkernel_batch
    kw = {k: part[k] for k in ("vp", "rho") if k in part}
    return depthkernel_batch(part["node_off"], part["depz"], part["vs"], part["per_off"],
                             part["periods"], minthk, form=form, **kw)


def run_sharded(node_off, depz, vs, per_off, periods, minthk, *, form=1, vp=None, rho=None,
                compute=None, group=None, dst: int = 0, device=None):
    """Run this rank's shard of a ragged batch and gather every rank's
    outputs to rank `dst` (torch.distributed: NCCL with device tensors, or
    gloo with host tensors).  Returns on `dst` the whole batch's outputs as
    tensors (keys pv, status, sen_vs, sen_vp, sen_rho, lsen, in
    dazi_dk_batch's layout, plus the offsets per_off, sen_off, ls_off) and
    None on the other ranks.  `compute(part, minthk, form)` runs one shard
    and returns arrays or tensors; the default is the GPU batch entry
    (dazi_dk_batch).  device: where the exchanged tensors live (default:
    the current CUDA device for NCCL, else the CPU)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if device is None:
        nccl = dist.get_backend(group) == "nccl"
        device = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
    node_off = np.asarray(node_off, np.int64)
    per_off = np.asarray(per_off, np.int64)
    bounds = shard_bounds(column_work(node_off, per_off, minthk), world)
    c0, c1 = int(bounds[rank]), int(bounds[rank + 1])
    part = slice_batch(node_off, depz, vs, per_off, periods, c0, c1, vp, rho)
    res = (compute or _default_compute)(part, minthk, form)
    def as_tensor(x):
        if x is None:
            return None
        t = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x))
        return t.to(device).reshape(-1)

    mine = {k: as_tensor(res.get(k)) for k in OUTPUT_KEYS}
    out = gather_blocks(mine, dst=dst, group=group)
    if out is None:
        return None
    sen_off, ls_off = output_offsets(node_off, per_off)
    out.update(per_off=per_off, sen_off=sen_off, ls_off=ls_off)
    return out
