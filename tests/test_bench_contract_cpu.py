"""bench.py's reference arm on the CPU: one JSON line with the keys a caller
of the benchmark reads (metric, value, unit, the CPU baseline block and an
e2e block with no host-device copies), on a tiny sample."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--ref-E", "2", "--n", "20", "--iters", "3"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "relaxations/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "relaxations/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "scaling", "vs_baseline", "dtype", "data",
                "config"):
        assert key in d


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--ref-E", "2", "--n", "20", "--iters", "3"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]


def test_plain_reference_driver_matches_oracle_lbfgs():
    """bench.py's plain form P runs the reference's own lbfgs (installed
    unmodified in baseline/_ref) through run_simulation_plain, the flow of
    pack_dynamics.OptimizerBFGS.run_simulation.  Driven by the FP64 oracle
    cost on CPU it must reproduce the oracle's lbfgs restatement: the
    flattening, the objective's buffers and the arguments are right."""
    import numpy as np
    import pytest
    import torch
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as O
    lbfgs_ref = bench.reference_lbfgs()
    if lbfgs_ref is None:
        pytest.skip("reference package not installed (baseline/install_ref.py)")
    E, n, iters, hist = 3, 10, 30, 5
    xyt, h = bench.workload(E, n, seed=4)

    def cost_fn(x, hh, c, g, gh):
        cc, gg, ghh = O.compound_cost(x.numpy(), hh.numpy(), w_area=1e-2, fixed_h=True)
        c.copy_(torch.from_numpy(cc))
        g.copy_(torch.from_numpy(gg))
        gh.copy_(torch.from_numpy(ghh))

    x, _ = bench.run_simulation_plain(lbfgs_ref, cost_fn, torch.from_numpy(xyt).double(),
                                      torch.from_numpy(h).double(), iters, hist)
    x0 = np.concatenate([xyt.reshape(E, -1), h], 1).astype(np.float64)

    def f(xx):
        c, g, gh = O.compound_cost(xx[:, :3 * n].reshape(E, n, 3), xx[:, 3 * n:], w_area=1e-2, fixed_h=True)
        return c, np.concatenate([g.reshape(E, -1), gh], 1)

    xo, _ = O.lbfgs(f, x0, max_iter=iters, history_size=hist, max_step=0.01, tolerance_grad=0, tolerance_change=0)
    np.testing.assert_allclose(x.numpy(), xo, rtol=0, atol=1e-10)


def test_roofline_work_constants_match_oracle_op_counts():
    """bench.py's algorithmic work per unit equals the oracle's op count of
    the reference arithmetic: cull, box tests, per-tree work, the average
    piece pair on the seeded 8 x n = 200 initial packings, and the lbfgs
    iteration (lbfgs_torch_parallel.py:531-724)."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as O
    x, _ = bench.workload(8, 200, seed=0)
    d = O.count_ops(x.astype(np.float64))
    assert d["pairs"] == 8 * 200 * 199 // 2 and d["trees"] == 1600
    assert d["ops_cull"] == bench.FLOPS_PER_PAIR * d["pairs"]
    assert d["ops_aabb"] == bench.FLOPS_PER_NEAR * d["near_pairs"]
    assert d["ops_tree"] + d["ops_boundary"] == bench.FLOPS_PER_TREE * d["trees"]
    assert round(d["ops_narrow"] / d["piece_pairs"]) == bench.FLOPS_PER_PIECE_PAIR
    N, m = 603, 10
    assert O.lbfgs_ops(N, m) == bench.FLOPS_PER_HIST_ELEM * N * m + bench.FLOPS_PER_ITER_ELEM * N
