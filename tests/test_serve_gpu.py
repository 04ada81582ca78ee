"""Continuous-batching service: results equal the one-shot relaxation, alone
and in a mix of other requests, whatever the chunking; admission respects the
memory pool."""
import numpy as np
import pytest
import torch

from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu


def _spec():
    from packing_b200.cost import CostSpec
    return CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)


def _job(n, seed):
    return poses(1, n, seed=seed)[0], square_h(1, n)[0]


def test_alone_equals_mix_equals_one_shot(cuda):
    from packing_b200.relax import RelaxParams, relax
    from packing_b200.serve import RelaxServer
    xA, hA = _job(57, 1)
    itA = 60
    s1 = RelaxServer(_spec(), history=6, chunk_iters=7, device=cuda)
    rA = s1.submit(xA, hA, itA)
    s1.drain()
    s2 = RelaxServer(_spec(), history=6, chunk_iters=13, device=cuda)
    others = [s2.submit(*_job(n, 10 + n), it) for n, it in [(200, 90), (12, 30), (120, 75), (33, 120)]]
    rA2 = s2.submit(xA, hA, itA)
    others += [s2.submit(*_job(n, 20 + n), it) for n, it in [(180, 50), (5, 20)]]
    s2.drain()
    assert np.array_equal(rA.result, rA2.result)
    assert rA.loss == rA2.loss and rA.iterations == rA2.iterations == itA
    # and equal to the single-launch relaxation with the same settings
    xo, ho, loss, it = relax(torch.from_numpy(xA[None]).to(cuda), torch.from_numpy(hA[None]).to(cuda), _spec(),
                             RelaxParams(n_iterations=itA, history_size=6, max_step=0.01, final_eval=True))
    assert np.array_equal(xo[0].cpu().numpy(), rA.result)
    assert float(loss[0]) == rA.loss
    for r in others:
        assert r.iterations == r.iters and np.isfinite(r.loss)


def test_memory_admission(cuda):
    from packing_b200.serve import RelaxServer
    srv = RelaxServer(_spec(), history=4, chunk_iters=5, device=cuda, pool_floats=1)
    foot = srv.footprint(100)
    srv = RelaxServer(_spec(), history=4, chunk_iters=5, device=cuda, pool_floats=2 * foot + 10)
    reqs = [srv.submit(*_job(100, k), 12) for k in range(5)]
    peak = 0
    while srv.pending or srv.resident:
        srv.step()
        peak = max(peak, len(srv.resident))
    assert peak <= 2
    assert all(r.iterations == 12 for r in reqs)
    with pytest.raises(ValueError):
        srv.submit(*_job(1000, 0), 5)


def test_trace_reports_latency(cuda):
    from packing_b200.serve import RelaxServer
    rng = np.random.default_rng(0)
    reqs = []
    for k in range(40):
        n = int(round(np.exp(rng.uniform(np.log(10), np.log(200)))))
        reqs.append((*_job(n, 100 + k), int(rng.integers(50, 301))))
    arrivals = np.cumsum(rng.exponential(0.002, size=len(reqs)))
    srv = RelaxServer(_spec(), history=10, chunk_iters=25, device=cuda)
    stats, done = srv.run_trace(reqs, arrivals)
    assert stats["requests"] == 40 and stats["p99_ms"] >= stats["p50_ms"] > 0
    assert all(r.iterations == r.iters for r in done)


def test_size_classes_do_not_change_results(cuda):
    """The engine's per-class launches give the bits of one launch over all
    resident jobs."""
    from packing_b200.serve import RelaxServer
    jobs = [(n, 30 + (7 * n) % 90) for n in (3, 9, 17, 25, 41, 66, 85, 120, 150, 199, 200, 250)]
    out = []
    for classes in (True, False):
        srv = RelaxServer(_spec(), history=5, chunk_iters=11, device=cuda, classes=classes)
        reqs = [srv.submit(*_job(n, 300 + n), it) for n, it in jobs]
        srv.drain()
        out.append(reqs)
    for a, b in zip(*out):
        assert np.array_equal(a.result, b.result) and np.array_equal(a.h_out, b.h_out)
        assert a.loss == b.loss and a.iterations == b.iterations
