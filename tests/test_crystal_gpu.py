"""Periodic (crystal) form of overlap_multi_ensemble against the FP64 oracle,
which reproduces the reference's recorded lattice values
(tests/test_oracle_golden.py): cost rtol 1e-5, gradient rtol = atol = 1e-4,
the reference's own FP32-vs-FP64 tolerances (pack_test.py:286-297)."""
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "cost_cases.json")


def _run(x, ax, use_sep, only_self, npd, dev):
    from packing_b200 import pack_cuda
    xt = torch.from_numpy(np.asarray(x, np.float32)).to(dev)
    at = torch.from_numpy(np.asarray(ax, np.float32)).to(dev)
    c = torch.empty(xt.shape[0], device=dev)
    g = torch.empty_like(xt)
    pack_cuda.overlap_multi_ensemble(xt, xt, use_sep, out_cost=c, out_grads=g, crystal_axes=at,
                                     only_self_interactions=only_self, N_periodic=npd)
    return c.cpu().numpy(), g.cpu().numpy()


@pytest.mark.parametrize("use_sep", [False, True])
@pytest.mark.parametrize("only_self", [False, True])
def test_lattice_golden_cases(cuda, use_sep, only_self):
    with open(GOLD) as f:
        d = json.load(f)
    rec = d["recorded_lattice"]
    key = "CollisionCostSeparation(scaling=5)" if use_sep else "CollisionCostOverlappingArea(scaling=3)"
    scale = 5.0 if use_sep else 3.0
    for k, cse in enumerate(d["lattice_cases"]):
        x = np.array(cse["xyt"], np.float32)[None]
        ax = np.array(cse["crystal_axes"], np.float32)[None]
        c, g = _run(x, ax, use_sep, only_self, cse["N_periodic"], cuda)
        oc, og = O.pair_cost_crystal(x.astype(np.float64), ax.astype(np.float64), use_sep, only_self,
                                     cse["N_periodic"])
        np.testing.assert_allclose(c, oc, rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(g, og, rtol=1e-4, atol=1e-4)
        if not only_self:
            # the reference's own FP32 GPU result (run_tests.ipynb) and its FP64 CPU value
            assert scale * c[0] == pytest.approx(rec[key]["cpu64"][k], rel=1e-5)
            assert scale * c[0] == pytest.approx(rec[key]["gpu32"][k], rel=2e-5)


@pytest.mark.parametrize("n,npd", [(5, 2), (12, 1), (3, 3)])
def test_random_lattices_vs_oracle(cuda, n, npd):
    rng = np.random.default_rng(n * 10 + npd)
    E = 16
    side = 0.9 * np.sqrt(n * 0.2456875)
    x = np.concatenate([rng.uniform(0, side, (E, n, 2)), rng.uniform(0, 2 * np.pi, (E, n, 1))], 2)
    ang = rng.uniform(np.pi / 3, 2 * np.pi / 3, E)
    a = side * rng.uniform(0.9, 1.1, E)
    b = side * rng.uniform(0.9, 1.1, E)
    ax = np.stack([a, np.zeros(E), b * np.cos(ang), b * np.sin(ang)], 1)
    x, ax = x.astype(np.float32), ax.astype(np.float32)
    for use_sep in (False, True):
        c, g = _run(x, ax, use_sep, False, npd, cuda)
        oc, og = O.pair_cost_crystal(x.astype(np.float64), ax.astype(np.float64), use_sep, False, npd)
        np.testing.assert_allclose(c, oc, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(g, og, rtol=1e-4, atol=1e-4)


def test_only_self_without_axes_is_zero(cuda):
    from packing_b200 import pack_cuda
    x = torch.rand((3, 4, 3), device=cuda)
    c = torch.ones(3, device=cuda)
    g = torch.ones_like(x)
    pack_cuda.overlap_multi_ensemble(x, x, False, out_cost=c, out_grads=g, only_self_interactions=True)
    assert float(c.abs().sum()) == 0.0 and float(g.abs().sum()) == 0.0


def test_batched_equals_single(cuda):
    """pack_test.py:418-445 property on the periodic path: bit-identical."""
    with open(GOLD) as f:
        d = json.load(f)
    cs = d["lattice_cases"][:3]
    x = np.stack([np.array(c["xyt"], np.float32) for c in cs])
    ax = np.stack([np.array(c["crystal_axes"], np.float32) for c in cs])
    cb, gb = _run(x, ax, False, False, 2, cuda)
    for k in range(3):
        c1, g1 = _run(x[k:k + 1], ax[k:k + 1], False, False, 2, cuda)
        assert np.array_equal(c1, cb[k:k + 1]) and np.array_equal(g1, gb[k:k + 1])
