"""Instance sharding: balanced partitions and the per-generation gather,
exercised with world_size 2 over gloo on CPU (no GPU involved)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from packing_b200.shard import gather_results, partition


def test_partition_balances_work():
    rng = np.random.default_rng(0)
    sizes = np.round(np.exp(rng.uniform(np.log(5), np.log(200), 1000))).astype(int)
    for world in (1, 2, 3, 8):
        parts = partition(sizes, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(sizes)
        assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
        work = [float((sizes[a:b].astype(float) ** 2).sum()) for a, b in parts]
        assert max(work) <= (sum(work) / world) * 1.05 + 200 ** 2
    assert partition([], 4) == [(0, 0)] * 4
    assert partition([10, 10], 4)[-1][1] == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ranges = partition(sizes, world)
        s, e = ranges[rank]
        # stand-in for the per-packing results of this rank's relaxation
        local = torch.stack([torch.arange(s, e, dtype=torch.float64),
                             torch.tensor(sizes[s:e], dtype=torch.float64) * 0.5,
                             torch.full((e - s,), float(rank), dtype=torch.float64)], 1)
        table = gather_results(local, [b - a for a, b in ranges])
        q.put((rank, table.numpy()))
    finally:
        dist.destroy_process_group()


def test_gather_results_two_ranks_gloo():
    sizes = [5, 200, 17, 64, 1, 120, 33]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ranges = partition(sizes, 2)
    for r in range(2):
        t = out[r]
        assert t.shape == (len(sizes), 3)
        assert np.array_equal(t[:, 0], np.arange(len(sizes)))
        assert np.array_equal(t[:, 1], np.array(sizes) * 0.5)
        owner = np.concatenate([[k] * (b - a) for k, (a, b) in enumerate(ranges)])
        assert np.array_equal(t[:, 2], owner)


def _champ_worker(rank, world, port, q):
    from packing_b200.shard import gather_champions
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        xyt, fit = _champ_population()
        ranges = [(0, 3), (3, 11)]   # rank 0 holds fewer packings than k
        s, e = ranges[rank]
        q.put((rank, [t.numpy() for t in gather_champions(xyt[s:e], fit[s:e], s, 5)]))
    finally:
        dist.destroy_process_group()


def _champ_population():
    g = torch.Generator().manual_seed(3)
    xyt = torch.rand((11, 4, 3), generator=g)
    fit = torch.tensor([0.5, 0.2, 0.9, 0.2, 0.7, 0.1, 0.2, 0.8, 0.3, float("inf"), 0.05])
    return xyt, fit


def test_gather_champions_two_ranks_gloo():
    """Every rank gets the same k best packings, ties to the lower global
    index, equal to selecting from the whole population in one process."""
    from packing_b200.shard import gather_champions
    xyt, fit = _champ_population()
    ref = gather_champions(xyt, fit, 0, 5)
    assert ref[2].tolist() == [10, 5, 1, 3, 6]
    assert torch.equal(ref[0], xyt[ref[2]])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_champ_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        for a, b in zip(out[r], ref):
            assert np.array_equal(a, b.numpy())
    # fewer packings than k in the whole population
    few = gather_champions(xyt[:2], fit[:2], 0, 5)
    assert few[2].tolist() == [1, 0]
