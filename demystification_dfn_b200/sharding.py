"""Placement of independent fault networks on the ranks of a job.

One process per GPU; networks never exchange data, so an ensemble shards by
whole networks and the only collective is the max-over-ranks of the timed
region (and the sum of the work done). Networks go to ranks greedily by
their K.V bytes (N^2, the per-stage cost), largest first, each to the rank
with the least work so far (ties to the lower rank), which keeps the
heaviest rank within one network of the mean.
"""
from __future__ import annotations


def shard_by_work(sizes, world, rank):
    """Indices of the networks (element counts ``sizes``) that ``rank`` of
    ``world`` integrates."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]) ** 2, i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += int(sizes[i]) ** 2
    return [i for i in range(len(sizes)) if owner[i] == rank]


def reduce_timing(ms_local, work_local, dist=None, device=None):
    """(max over ranks of the timed milliseconds, sum over ranks of the work):
    whole-job throughput is sum(work) / max(ms). Without a process group the
    local values are returned."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms_local), float(work_local)
    import torch

    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    w = torch.tensor([float(work_local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
