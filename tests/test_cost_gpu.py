"""CUDA cost kernels against the FP64 oracle and the reference's recorded
values.  Tolerances are the reference's own FP32-vs-FP64 test tolerances
(core/pack_test.py:286-297): cost rtol 1e-5, gradient rtol = atol = 1e-4."""
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
RTOL_COST, TOL_GRAD = 1e-5, 1e-4


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def _overlap(x, use_sep, dev, grad=True):
    from packing_b200 import pack_cuda
    xt = _t(x, dev)
    c = torch.empty(x.shape[0], device=dev)
    g = torch.empty_like(xt) if grad else None
    pack_cuda.overlap_multi_ensemble(xt, xt, use_sep, out_cost=c, out_grads=g)
    return c.cpu().numpy(), (g.cpu().numpy() if grad else None)


def _boundary(x, h, dev):
    from packing_b200 import pack_cuda
    xt, ht = _t(x, dev), _t(h, dev)
    c = torch.empty(x.shape[0], device=dev)
    g = torch.empty_like(xt)
    gh = torch.empty_like(ht)
    pack_cuda.boundary_distance_multi_ensemble(xt, ht, out_cost=c, out_grads=g, out_grad_h=gh)
    return c.cpu().numpy(), g.cpu().numpy(), gh.cpu().numpy()


def _golden():
    with open(os.path.join(GOLD, "cost_cases.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("k", range(4))
def test_golden_cases(cuda, k):
    d = _golden()
    case = d["cases"][k]
    rec = d["recorded"]
    x = np.array(case["xyt"])[None]
    h = np.array([case["h"]])
    # overlap area x3
    c, g = _overlap(x, False, cuda)
    assert 3 * c[0] == pytest.approx(rec["CollisionCostOverlappingArea(scaling=3)"]["cpu64"][k], rel=RTOL_COST)
    oc, og = O.pair_cost(x.astype(np.float32).astype(np.float64), False)
    np.testing.assert_allclose(g, og, rtol=TOL_GRAD, atol=TOL_GRAD)
    # separation x5
    c, g = _overlap(x, True, cuda)
    assert 5 * c[0] == pytest.approx(rec["CollisionCostSeparation(scaling=5)"]["cpu64"][k], rel=RTOL_COST)
    oc, og = O.pair_cost(x.astype(np.float32).astype(np.float64), True)
    np.testing.assert_allclose(g, og, rtol=TOL_GRAD, atol=TOL_GRAD)
    # boundary x1 / x5
    c, g, gh = _boundary(x, h, cuda)
    assert c[0] == pytest.approx(rec["BoundaryDistanceCost(use_kernel=False)"]["cpu64"][k], rel=RTOL_COST)
    assert 5 * c[0] == pytest.approx(rec["BoundaryDistanceCost(use_kernel=True, scaling=5)"]["cpu64"][k],
                                     rel=RTOL_COST)
    ob, obg, obh = O.boundary(x.astype(np.float32).astype(np.float64), h.astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(g, obg, rtol=TOL_GRAD, atol=TOL_GRAD)
    np.testing.assert_allclose(gh, obh, rtol=TOL_GRAD, atol=TOL_GRAD)
    # CostCompound(scaling 1.5, [AreaCost, Separation]) through the fused kernel
    from packing_b200.cost import CostSpec, compound_cost
    spec = CostSpec(pair="sep", w_pair=1.5, w_boundary=0.0, w_area=1.5, fixed_h=False)
    cc, gg, ggh = compound_cost(_t(x, cuda), _t(h, cuda), spec)
    assert float(cc[0]) == pytest.approx(
        rec["CostCompound(scaling=1.5, [AreaCost, CollisionCostSeparation])"]["cpu64"][k], rel=RTOL_COST)
    np.testing.assert_allclose(ggh.cpu().numpy(), [[1.5 * 2 * h[0, 0], 0, 0]], rtol=1e-6)


@pytest.mark.parametrize("use_sep", [False, True])
def test_config1_workload_vs_oracle(cuda, use_sep):
    """64 packings of n=20 (the CPU-reference configuration)."""
    x = poses(64, 20, seed=0)
    c, g = _overlap(x, use_sep, cuda)
    oc, og = O.pair_cost(x.astype(np.float64), use_sep)
    np.testing.assert_allclose(c, oc, rtol=RTOL_COST, atol=1e-6)
    np.testing.assert_allclose(g, og, rtol=TOL_GRAD, atol=TOL_GRAD)


@pytest.mark.parametrize("use_sep", [False, True])
def test_n200_vs_oracle(cuda, use_sep):
    x = poses(6, 200, seed=1)
    c, g = _overlap(x, use_sep, cuda)
    oc, og = O.pair_cost(x.astype(np.float64), use_sep)
    np.testing.assert_allclose(c, oc, rtol=RTOL_COST, atol=1e-6)
    np.testing.assert_allclose(g, og, rtol=TOL_GRAD, atol=TOL_GRAD)


def test_forward_only_equals_with_gradient_bitwise(cuda):
    """pack_test.py:268-271: cost without gradient == cost with gradient."""
    x = poses(32, 50, seed=4)
    for sep in (False, True):
        c1, _ = _overlap(x, sep, cuda, grad=True)
        c2, _ = _overlap(x, sep, cuda, grad=False)
        assert np.array_equal(c1, c2)


def test_batched_equals_single_bitwise(cuda):
    """pack_test.py:372-447: a packing's result does not depend on the batch."""
    x = poses(12, 40, seed=5)
    for sep in (False, True):
        cb, gb = _overlap(x, sep, cuda)
        for e in (0, 5, 11):
            cs, gs = _overlap(x[e:e + 1], sep, cuda)
            assert np.array_equal(cb[e:e + 1], cs)
            assert np.array_equal(gb[e:e + 1], gs)


def test_ragged_equals_uniform_bitwise(cuda):
    from packing_b200.cost import CostSpec, compound_cost
    sizes = [7, 31, 1, 64, 20, 0, 128]
    xs = [poses(1, n, seed=10 + n)[0] for n in sizes]
    hs = np.concatenate([square_h(1, max(n, 1)) for n in sizes])
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=0.0)
    flat = np.concatenate([a.reshape(-1, 3) for a in xs]) if sum(sizes) else np.zeros((0, 3), np.float32)
    offs = torch.tensor(np.concatenate([[0], np.cumsum(sizes)]), dtype=torch.int32, device=cuda)
    cr, gr, ghr = compound_cost(_t(flat, cuda), _t(hs, cuda), spec, offsets=offs, n_max=max(sizes))
    o = np.concatenate([[0], np.cumsum(sizes)])
    for e, n in enumerate(sizes):
        cu, gu, ghu = compound_cost(_t(xs[e][None], cuda), _t(hs[e:e + 1], cuda), spec)
        assert float(cr[e]) == float(cu[0]) or (n == 0 and float(cr[e]) == 0.0)
        assert np.array_equal(gr[o[e]:o[e + 1]].cpu().numpy(), gu[0].cpu().numpy())


def test_compound_matches_oracle(cuda):
    """OptimizerBFGS default cost (pack_dynamics.py:45-51) at n=200."""
    from packing_b200.cost import CostSpec, compound_cost
    x = poses(4, 200, seed=2)
    h = square_h(4, 200)
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)
    c, g, gh = compound_cost(_t(x, cuda), _t(h, cuda), spec)
    oc, og, ogh = O.compound_cost(x.astype(np.float64), h.astype(np.float64), w_area=1e-2, fixed_h=True)
    np.testing.assert_allclose(c.cpu().numpy(), oc, rtol=RTOL_COST)
    np.testing.assert_allclose(g.cpu().numpy(), og, rtol=TOL_GRAD, atol=TOL_GRAD)
    assert np.all(gh.cpu().numpy() == 0)


def test_edge_cases(cuda):
    from packing_b200 import pack_cuda
    # empty batch, zero and one tree
    for shape in [(0, 5, 3), (3, 0, 3), (3, 1, 3)]:
        x = torch.zeros(shape, device=cuda)
        c = torch.full((shape[0],), 7.0, device=cuda)
        g = torch.full(shape, 7.0, device=cuda)
        pack_cuda.overlap_multi_ensemble(x, x, False, out_cost=c, out_grads=g)
        assert torch.all(c == 0) and torch.all(g == 0)
    # identical poses: the overlap is the whole tree, gradients cancel by symmetry
    x = np.zeros((1, 2, 3), np.float32)
    x[0, :, 2] = 0.3
    c, g = _overlap(x, False, cuda)
    _, _, _, _, _, area = O.geometry()
    assert c[0] == pytest.approx(area, rel=1e-5)
    oc, og = O.pair_cost(x.astype(np.float64), False)
    assert oc[0] == pytest.approx(area, rel=1e-9)
    # far apart: nothing
    x = np.array([[[0, 0, 0], [5, 0, 1.0]]], np.float32)
    c, g = _overlap(x, False, cuda)
    assert c[0] == 0 and np.all(g == 0)
    # maximum size and one beyond
    x = poses(1, 1024, seed=9)
    c, g = _overlap(x, False, cuda)
    oc, og = O.pair_cost(x.astype(np.float64), False)
    np.testing.assert_allclose(c, oc, rtol=RTOL_COST)
    with pytest.raises(ValueError):
        _overlap(poses(1, 1025, seed=9), False, cuda)


@pytest.mark.parametrize("layout", ["cluster", "line", "spread", "cluster1024"])
def test_broad_phase_layouts_vs_oracle(cuda, layout):
    """Layouts that stress the cell grid: every pair near (the near list is
    written in many chunks), a single row of cells, an extent far larger than
    the grid (cells grow), and the maximum size fully clustered."""
    rng = np.random.default_rng(11)
    if layout == "cluster":
        n = 300
        x = np.concatenate([rng.uniform(-0.15, 0.15, (1, n, 2)), rng.uniform(0, 6.3, (1, n, 1))], axis=2)
    elif layout == "line":
        n = 400
        x = np.stack([np.arange(n) * 0.3, rng.uniform(-0.05, 0.05, n), rng.uniform(0, 6.3, n)], axis=1)[None]
    elif layout == "spread":
        n = 256
        x = np.concatenate([rng.uniform(-1000, 1000, (1, n, 2)), rng.uniform(0, 6.3, (1, n, 1))], axis=2)
        x[0, 1::2, :2] = x[0, 0::2, :2] + rng.uniform(-0.4, 0.4, (n // 2, 2))   # overlapping pairs
    else:
        n = 1024
        x = np.concatenate([rng.uniform(-0.5, 0.5, (1, n, 2)), rng.uniform(0, 6.3, (1, n, 1))], axis=2)
    x = x.astype(np.float32)
    # 1024 trees in a unit square: every tree overlaps ~1000 others, many of
    # them nearly coincident, and float32 clipping of such pairs is
    # ill-conditioned; a missed or doubled pair would still move a gradient
    # by O(0.1), far above this bound
    tol = 1e-2 if layout == "cluster1024" else TOL_GRAD
    for use_sep in (False, True):
        c, g = _overlap(x, use_sep, cuda)
        oc, og = O.pair_cost(x.astype(np.float64), use_sep)
        np.testing.assert_allclose(c, oc, rtol=RTOL_COST, atol=1e-6)
        np.testing.assert_allclose(g, og, rtol=TOL_GRAD, atol=tol)
        assert float(np.abs(g - og).mean()) < TOL_GRAD


def test_argument_errors(cuda):
    from packing_b200 import pack_cuda
    x = torch.zeros((2, 4, 3), device=cuda)
    c = torch.zeros(2, device=cuda)
    with pytest.raises(ValueError):
        pack_cuda.overlap_multi_ensemble(x.double(), x.double(), False, out_cost=c.double())
    with pytest.raises(ValueError):
        pack_cuda.overlap_multi_ensemble(x, x, False, out_cost=torch.zeros(3, device=cuda))
    with pytest.raises(NotImplementedError):
        pack_cuda.overlap_multi_ensemble(x, x.clone(), False, out_cost=c)
    with pytest.raises(ValueError):   # crystal axes must be (E, 4)
        pack_cuda.overlap_multi_ensemble(x, x, False, out_cost=c, crystal_axes=torch.zeros(3, 4, device=cuda))
    with pytest.raises(ValueError):
        pack_cuda.overlap_multi_ensemble(x, x, False, out_cost=c, crystal_axes=torch.zeros(2, 4, device=cuda),
                                         N_periodic=-1)
