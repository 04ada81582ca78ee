"""Instance sharding across GPUs (one process per GPU, torch.distributed).

Packings are independent, so the path shards by instance with no collective
in the data path (the reference itself runs on one GPU and has no distribution).
A GA generation needs one small exchange afterwards -- every rank learns the
per-packing results (loss, square side, iterations) of all ranks -- which is
one all_gather of a few floats per packing.

``partition(sizes, world)`` splits instances into contiguous, work-balanced
ranges (work ~ n^2 per packing: the pair enumeration and the near pairs grow
with n^2 at fixed density).  ``gather_results(local, counts, group)``
all-gathers per-instance rows of the shards into the global order.
``relax_shard(...)`` relaxes this rank's range with the fused kernel.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def partition(sizes, world: int):
    """Contiguous ranges [(start, end)] per rank, balancing sum(n^2)."""
    sizes = np.asarray(sizes, dtype=np.float64)
    E = len(sizes)
    if world <= 1 or E == 0:
        return [(0, E)] + [(E, E)] * max(0, world - 1)
    w = np.cumsum(sizes ** 2)
    total = w[-1]
    cuts = [0]
    for r in range(1, world):
        k = int(np.searchsorted(w, total * r / world, side="left")) + 1
        cuts.append(min(max(k, cuts[-1]), E))
    cuts.append(E)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def gather_results(local: torch.Tensor, counts, group=None) -> torch.Tensor:
    """local: (count_rank, k) rows of this rank; counts: rows per rank.
    Returns the (sum counts, k) concatenation in rank order on every rank."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    k = local.shape[1]
    mx = max(counts) if counts else 0
    buf = torch.zeros((mx, k), dtype=local.dtype, device=local.device)
    buf[:counts[rank]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][:counts[r]] for r in range(world)], dim=0)


def relax_shard(xyt_list, h, spec, params, rank: int, world: int, device=None, group=None):
    """Relax this rank's share of a ragged population in one launch and
    return the all-gathered per-packing (loss, side of h, iterations) table
    together with this rank's relaxed packings and range."""
    from .relax import relax_ragged
    sizes = [int(a.shape[0]) for a in xyt_list]
    ranges = partition(sizes, world)
    s, e = ranges[rank]
    dev = torch.device(device or "cuda")
    mine = [torch.as_tensor(a, device=dev) for a in xyt_list[s:e]]
    hh = torch.as_tensor(h[s:e], device=dev)
    if mine:
        outs, ho, loss, it = relax_ragged(mine, hh, spec, params)
        local = torch.stack([loss.double(), ho[:, 0].double(), it.double()], 1)
    else:
        outs, local = [], torch.zeros((0, 3), dtype=torch.float64, device=dev)
    if world > 1:
        table = gather_results(local, [b - a for a, b in ranges], group)
    else:
        table = local
    return table, outs, (s, e)
