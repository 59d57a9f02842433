"""Sharding of independent trajectories over ranks (one process per GPU).

Trajectories never exchange data, so a batch splits by rows with no collective
on the solver's data path.  ``partition_rows`` balances rows by their work
(n * steps for a ragged batch) with a deterministic longest-first greedy
assignment, so every rank computes the same partition without communication.
``gather_rows`` and ``max_over_ranks`` assemble results (optional) and take the
max over ranks of device times for benchmarking.  Data-parallel training of a
corrector has one real exchange per step: ``average_gradients_`` averages the
network's gradients over the ranks (what DDP does; weighted by each rank's rows
when the shards are unequal), one all-reduce of one flat bucket.
"""
from __future__ import annotations

import heapq

import torch


def partition_rows(work, world: int):
    """Row indices per rank, balanced by `work` (longest first onto the lightest rank).

    Deterministic for a given `work`; returns `world` sorted index lists."""
    if world <= 0:
        raise ValueError("world must be positive")
    work = [float(w) for w in work]
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(p) for p in parts]


def contiguous_rows(rows: int, rank: int, world: int) -> range:
    """The contiguous block of a uniform batch owned by `rank`."""
    per, extra = divmod(rows, world)
    start = rank * per + min(rank, extra)
    return range(start, start + per + (1 if rank < extra else 0))


def gather_rows(local: torch.Tensor, parts, rank: int, world: int, group=None) -> torch.Tensor:
    """Reassemble a [rows, ...] tensor from every rank's rows (indices `parts`)."""
    import torch.distributed as dist
    width = max(len(p) for p in parts)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    rows = sum(len(p) for p in parts)
    out = torch.empty((rows,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r, p in enumerate(parts):
        if p:
            out[torch.as_tensor(p, device=local.device)] = bufs[r][: len(p)]
    return out


def max_over_ranks(value: float, device=None, group=None) -> float:
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def allreduce_mean_(tensors, group=None) -> None:
    """Average `tensors` in place over the ranks of `group`: the values are packed into one
    flat bucket, summed by one all-reduce and divided by the world size.  Every rank must pass
    tensors of the same shapes in the same order (a None entry raises ValueError: its length
    would differ between ranks); for parameter gradients use ``average_gradients_``."""
    import torch.distributed as dist
    ts = list(tensors)
    if any(t is None for t in ts):
        raise ValueError("allreduce_mean_: None entry (use average_gradients_ for parameter gradients)")
    if not ts or not dist.is_available() or not dist.is_initialized():
        return
    world = dist.get_world_size(group)
    if world == 1:
        return
    flat = torch.cat([t.reshape(-1) for t in ts])
    dist.all_reduce(flat, group=group)
    flat.div_(world)
    _unpack(flat, ts)


def _unpack(flat, ts):
    off = 0
    for t in ts:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n


def average_gradients_(params, group=None, local_rows=None) -> None:
    """Data-parallel gradient exchange for a corrector network: one all-reduce of one flat
    bucket per call, between ``backward()`` and the optimizer step.

    Every rank passes the same parameters in the same order.  A parameter whose gradient
    is None on this rank enters the bucket as zeros (and receives the averaged gradient),
    so the bucket has the same length on every rank whichever parameters took part in
    this rank's loss.

    ``local_rows`` (this rank's number of trajectories): each rank's loss is a mean over
    its own rows, so with unequal shards the plain average of the ranks' gradients weights
    rows unequally.  Given ``local_rows``, each rank's gradient is weighted by its rows and
    the sum divided by the total (all-reduced in the same bucket), which gives the gradient
    of the mean loss over all ranks' rows, as one process with the whole batch would.
    Without it the gradients are averaged over ranks (DDP's rule, exact for equal shards)."""
    import torch.distributed as dist
    ps = [p for p in params]
    if not ps or not dist.is_available() or not dist.is_initialized():
        return
    world = dist.get_world_size(group)
    if world == 1:
        return
    grads = []
    for p in ps:
        if p.grad is None:
            p.grad = torch.zeros_like(p)
        grads.append(p.grad)
    parts = [g.reshape(-1) for g in grads]
    if local_rows is not None:
        w = float(local_rows)
        parts = [g * w for g in parts] + [torch.full((1,), w, dtype=grads[0].dtype, device=grads[0].device)]
    flat = torch.cat(parts)
    dist.all_reduce(flat, group=group)
    if local_rows is not None:
        flat = flat[:-1] / flat[-1:]
    else:
        flat.div_(world)
    _unpack(flat, grads)
