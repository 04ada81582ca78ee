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
``gather_champions(xyt, fitness, offset, k, group)`` gives every rank the
same k best packings of the whole population (the reference set of the GA's
diversity matching, ``kaggle_support.py:2014-2129``) from one all_gather of
each rank's own k best.
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
    # gloo gathers host tensors: a CUDA table goes through host memory there
    # (NCCL gathers it in place)
    via_host = local.is_cuda and dist.get_backend(group) == "gloo"
    dev = torch.device("cpu") if via_host else local.device
    buf = torch.zeros((mx, k), dtype=local.dtype, device=dev)
    buf[:counts[rank]] = local.to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][:counts[r]] for r in range(world)], dim=0).to(local.device)


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


def gather_champions(xyt: torch.Tensor, fitness: torch.Tensor, offset: int, k: int, group=None):
    """The k packings of lowest fitness over all ranks, identical on every rank.

    xyt: (E_local, n, 3) this rank's packings (n equal on every rank);
    fitness: (E_local,); offset: global index of this rank's first packing.
    Each rank offers its own k best (ties to the lower global index), so one
    all_gather of k rows of (fitness, global index, n * 3 poses) in float64
    carries every candidate; the global selection uses the same order.
    Returns (xyt (k', n, 3) in xyt's dtype, fitness (k',) float64, global
    indices (k',) int64), k' = min(k, population size), best first.
    """
    if xyt.dim() != 3 or xyt.shape[2] != 3:
        raise ValueError("xyt must be (E_local, n, 3)")
    if fitness.shape != (xyt.shape[0],):
        raise ValueError("fitness must be (E_local,)")
    if k < 0:
        raise ValueError("k must be >= 0")
    E, n = xyt.shape[0], xyt.shape[1]
    dev = xyt.device
    fit = fitness.to(torch.float64)
    gidx = torch.arange(offset, offset + E, dtype=torch.float64, device=dev)

    def best(f, g, m):
        # lexicographic (fitness, global index): sort by index, then a stable sort by fitness
        o = torch.argsort(g, stable=True)
        o = o[torch.argsort(f[o], stable=True)]
        return o[:m]

    pick = best(fit, gidx, min(k, E))
    rows = torch.full((k, 2 + 3 * n), float("nan"), dtype=torch.float64, device=dev)
    rows[:, 0] = float("inf")
    rows[:, 1] = -1.0
    m = pick.numel()
    rows[:m, 0] = fit[pick]
    rows[:m, 1] = gidx[pick]
    rows[:m, 2:] = xyt[pick].reshape(m, 3 * n).to(torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        host = rows.is_cuda and dist.get_backend(group) == "gloo"   # gloo gathers host tensors
        buf = rows.cpu() if host else rows
        parts = [torch.empty_like(buf) for _ in range(dist.get_world_size(group))]
        dist.all_gather(parts, buf, group=group)
        rows = torch.cat(parts, 0).to(dev)
    rows = rows[rows[:, 1] >= 0]
    sel = best(rows[:, 0], rows[:, 1], min(k, rows.shape[0]))
    out = rows[sel]
    return (out[:, 2:].reshape(-1, n, 3).to(xyt.dtype), out[:, 0].clone(), out[:, 1].to(torch.int64))
