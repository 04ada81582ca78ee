"""The FP64 oracle against the reference's recorded golden values and its own
lbfgs -- the pins that make the oracle trustworthy (CPU only)."""
import itertools
import json
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O
from oracle.refsrc import reference_core

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _cases():
    with open(os.path.join(GOLD, "cost_cases.json")) as f:
        return json.load(f)


def test_geometry_constants():
    # kaggle_support.py:241-354: radius and area of the expanded tree
    pxy, pnv, txy, R, cut, area = O.geometry()
    assert list(pnv) == [3, 4, 4, 4]
    assert abs(R - 0.5796198151417984) < 1e-15
    assert abs(cut - (2 * R) ** 2) < 1e-15
    assert abs(area - 0.2456875) < 1e-6
    # pieces are CCW and tile the outline: their areas add up to the tree area
    tot = 0.0
    for p in range(4):
        v = pxy[p, :pnv[p]]
        s = 0.5 * np.sum(v[:, 0] * np.roll(v[:, 1], -1) - np.roll(v[:, 0], -1) * v[:, 1])
        assert s > 0
        tot += s
    assert abs(tot - area) < 1e-12


@pytest.mark.parametrize("k", range(4))
def test_costs_match_reference_fp64(k):
    """Oracle reproduces the reference's FP64 CPU values (run_tests.ipynb)."""
    d = _cases()
    c = d["cases"][k]
    x = np.array(c["xyt"])[None]
    h = np.array([c["h"]])
    rec = d["recorded"]
    ov = O.pair_cost(x, False)[0][0] * 3
    sp = O.pair_cost(x, True)[0][0] * 5
    b = O.boundary(x, h)[0][0]
    cc = 1.5 * (O.pair_cost(x, True)[0][0] + h[0, 0] ** 2)
    assert ov == pytest.approx(rec["CollisionCostOverlappingArea(scaling=3)"]["cpu64"][k], rel=1e-13)
    assert sp == pytest.approx(rec["CollisionCostSeparation(scaling=5)"]["cpu64"][k], rel=1e-13)
    assert b == pytest.approx(rec["BoundaryDistanceCost(use_kernel=False)"]["cpu64"][k], rel=1e-13)
    assert 5 * b == pytest.approx(rec["BoundaryDistanceCost(use_kernel=True, scaling=5)"]["cpu64"][k], rel=1e-13)
    assert cc == pytest.approx(rec["CostCompound(scaling=1.5, [AreaCost, CollisionCostSeparation])"]["cpu64"][k],
                               rel=1e-13)


def _fd(f, x, eps=1e-6):
    g = np.zeros_like(x)
    for idx in np.ndindex(x.shape):
        xp, xm = x.copy(), x.copy()
        xp[idx] += eps
        xm[idx] -= eps
        g[idx] = (f(xp) - f(xm)) / (2 * eps)
    return g


@pytest.mark.parametrize("use_sep", [False, True])
def test_oracle_gradient_matches_finite_differences(use_sep):
    """pack_test.py:301-370 check, on the oracle's analytic gradient."""
    x = O.place_random(10, 1.5, 0)[None]
    c, g = O.pair_cost(x, use_sep)
    fd = _fd(lambda xx: O.pair_cost(xx, use_sep)[0][0], x)
    np.testing.assert_allclose(g, fd, rtol=1e-4, atol=1e-4)
    h = np.array([[0.5, 0.2, 0.4]])
    cb, gb, ghb = O.boundary(x, h)
    fdb = _fd(lambda xx: O.boundary(xx, h)[0][0], x)
    np.testing.assert_allclose(gb, fdb, rtol=1e-4, atol=1e-4)
    fdh = _fd(lambda hh: O.boundary(x, hh)[0][0], h)
    np.testing.assert_allclose(ghb, fdh, rtol=1e-4, atol=1e-4)


def test_oracle_lbfgs_matches_reference_fixture():
    d = np.load(os.path.join(GOLD, "lbfgs_ref.npz"))
    A, b = d["A"], d["b"]

    def quad(x):
        Ax = np.einsum("mij,mj->mi", A, x)
        return 0.5 * (x * Ax).sum(1) - (b * x).sum(1), Ax - b

    x, _ = O.lbfgs(quad, d["x0_quad"], max_iter=15, history_size=5, max_step=0.5, tolerance_grad=0,
                   tolerance_change=0)
    np.testing.assert_allclose(x, d["x_quad"], rtol=0, atol=1e-12)
    n, E = int(d["n_pack"]), 3

    def pack(x):
        c, g, gh = O.compound_cost(x[:, :3 * n].reshape(E, n, 3), x[:, 3 * n:], w_area=1e-2, fixed_h=True)
        return c, np.concatenate([g.reshape(E, -1), gh], 1)

    x, _ = O.lbfgs(pack, d["x0_pack"], max_iter=25, history_size=3, max_step=0.01, tolerance_grad=0,
                   tolerance_change=0)
    np.testing.assert_allclose(x, d["x_pack"], rtol=0, atol=1e-10)


REF = reference_core()


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_oracle_lbfgs_matches_reference_live():
    """Against the reference module itself, with tolerances and history limits
    that exercise the shift and the stop tests."""
    sys.path.insert(0, REF)
    import torch
    import lbfgs_torch_parallel as R
    rng = np.random.default_rng(3)
    M, N = 5, 9
    A = rng.normal(size=(M, N, N))
    A = A @ A.transpose(0, 2, 1) + np.eye(N)[None]
    b = rng.normal(size=(M, N))
    x0 = rng.normal(size=(M, N)) * 3

    def quad(x):
        Ax = np.einsum("mij,mj->mi", A, x)
        return 0.5 * (x * Ax).sum(1) - (b * x).sum(1), Ax - b

    for kw in [dict(max_iter=40, history_size=3, max_step=0.3, tolerance_grad=1e-6, tolerance_change=1e-9),
               dict(max_iter=12, history_size=20, max_step=None, tolerance_grad=0, tolerance_change=0, lr=0.5),
               dict(max_iter=30, history_size=4, max_step=1.0, stop_on_cost_increase=True,
                    tolerance_rel_change=1e-3)]:
        xt = torch.from_numpy(x0.copy())
        R.lbfgs(lambda x, m: tuple(torch.from_numpy(a) for a in quad(x.numpy())), xt, **kw)
        xo, _ = O.lbfgs(quad, x0, **kw)
        np.testing.assert_allclose(xo, xt.numpy(), rtol=0, atol=1e-11)


def _brute_lap(C):
    n = C.shape[0]
    best, arg = None, None
    for perm in itertools.permutations(range(n)):
        s = sum(C[i, perm[i]] for i in range(n))
        if best is None or s < best:
            best, arg = s, perm
    return best, arg


def test_oracle_hungarian_optimal():
    from scipy.optimize import linear_sum_assignment
    rng = np.random.default_rng(0)
    for n in [1, 2, 3, 5, 7]:
        C = rng.random((6, n, n)).astype(np.float32)
        rm, tot = O.hungarian(C)
        for b in range(6):
            best, _ = _brute_lap(C[b].astype(np.float64))
            assert sorted(rm[b].tolist()) == list(range(n))
            assert abs(float(C[b][np.arange(n), rm[b]].astype(np.float64).sum()) - best) < 1e-5
    C = rng.random((20, 60, 60)).astype(np.float32)
    rm, tot = O.hungarian(C)
    for b in range(20):
        r, c = linear_sum_assignment(C[b].astype(np.float64))
        assert abs(C[b][r, c].astype(np.float64).sum() - C[b][np.arange(60), rm[b]].astype(np.float64).sum()) < 1e-4


@pytest.mark.parametrize("k", range(4))
def test_periodic_costs_match_reference_fp64(k):
    """Oracle's periodic form reproduces the reference's FP64 CPU values for
    the lattice solutions of pack_test.py:174-213 (run_tests.ipynb)."""
    d = _cases()
    c = d["lattice_cases"][k]
    x = np.array(c["xyt"])[None]
    ax = np.array(c["crystal_axes"])[None]
    rec = d["recorded_lattice"]
    ov = O.pair_cost_crystal(x, ax, False, False, c["N_periodic"])[0][0] * 3
    sp = O.pair_cost_crystal(x, ax, True, False, c["N_periodic"])[0][0] * 5
    assert ov == pytest.approx(rec["CollisionCostOverlappingArea(scaling=3)"]["cpu64"][k], rel=1e-13)
    assert sp == pytest.approx(rec["CollisionCostSeparation(scaling=5)"]["cpu64"][k], rel=1e-13)


@pytest.mark.parametrize("use_sep", [False, True])
def test_periodic_gradient_matches_finite_differences(use_sep):
    """The periodic ref-pose gradient (self images excluded, as in the
    reference) against central differences of the cost without the
    self-image terms' theta dependence: x, y derivatives match in full."""
    d = _cases()
    c = d["lattice_cases"][0]
    x = np.array(c["xyt"])[None]
    ax = np.array(c["crystal_axes"])[None]
    _, g = O.pair_cost_crystal(x, ax, use_sep, False, 2)
    fd = _fd(lambda xx: O.pair_cost_crystal(xx, ax, use_sep, False, 2)[0][0], x)
    # self images do not depend on a tree's own translation, so x, y agree
    np.testing.assert_allclose(g[..., :2], fd[..., :2], rtol=1e-4, atol=1e-4)
    # theta: the reference adds the self-image part by finite differences of
    # the only_self cost (pack_cost.py:636-672); together they match
    fd_self = _fd(lambda xx: O.pair_cost_crystal(xx, ax, use_sep, True, 2)[0][0], x)
    np.testing.assert_allclose(g[..., 2] + fd_self[..., 2] / 2, fd[..., 2], rtol=1e-4, atol=1e-4)
