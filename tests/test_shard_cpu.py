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
