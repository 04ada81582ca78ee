"""Instance sharding on the GPU: two ranks (gloo for the one exchange, both
on cuda:0 -- their kernels never wait on one another) each relax their
work-balanced share of one seeded ragged population with relax_shard.  The
gathered per-packing table and each rank's relaxed packings equal one
process's relax_ragged of the whole population, bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu


def _population():
    rng = np.random.default_rng(17)
    sizes = [int(round(np.exp(rng.uniform(np.log(5), np.log(90))))) for _ in range(24)]
    xs = [poses(1, n, seed=500 + k)[0] for k, n in enumerate(sizes)]
    h = np.concatenate([square_h(1, n) for n in sizes])
    return sizes, xs, h


def _spec_params():
    from packing_b200.cost import CostSpec
    from packing_b200.relax import RelaxParams
    return (CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True),
            RelaxParams(n_iterations=40, history_size=6, max_step=0.01))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from packing_b200 import _lib
    from packing_b200.shard import relax_shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        _lib.ensure_init(0)
        sizes, xs, h = _population()
        spec, prm = _spec_params()
        table, outs, rng = relax_shard(xs, h, spec, prm, rank, world, device="cuda:0")
        torch.cuda.synchronize()
        q.put((rank, table.cpu().numpy(), [o.cpu().numpy() for o in outs], rng))
    finally:
        dist.destroy_process_group()


def test_relax_shard_two_ranks_equals_one_process(cuda):
    from packing_b200.relax import relax_ragged
    from packing_b200.shard import partition
    sizes, xs, h = _population()
    spec, prm = _spec_params()
    outs, ho, loss, it = relax_ragged([torch.from_numpy(x).to(cuda) for x in xs], torch.from_numpy(h).to(cuda),
                                      spec, prm)
    ref_table = torch.stack([loss.double(), ho[:, 0].double(), it.double()], 1).cpu().numpy()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r, (t, o, g)) for r, t, o, g in (q.get(timeout=300) for _ in range(2)))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ranges = partition(sizes, 2)
    assert ranges[0][1] > 0 and ranges[1][1] - ranges[1][0] > 0   # both ranks hold packings
    for r in range(2):
        table, mine, rng = got[r]
        assert tuple(rng) == ranges[r]
        assert np.array_equal(table, ref_table)
        for k, o in zip(range(*rng), mine):
            assert np.array_equal(o, outs[k].cpu().numpy())
