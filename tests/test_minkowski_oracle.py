"""The exact-separation oracle (CPU restatement of core/pack_minkowski.py)
checked against facts that do not use its Minkowski machinery:

* outside the forbidden zone the value is minus the distance between the
  two tree polygons (dist(t, A - B) = dist(A, B + t));
* its inside test agrees with the overlap-area oracle (pack_cuda.py's
  area kernel restated in C);
* inside, no boundary point is nearer than the value along any ray, and
  one is found that near (penetration depth as the smallest exit distance).
"""
import math

import numpy as np
import pytest

from oracle import minkowski as MK
from oracle import oracle as O

THETAS = np.array([-math.pi, -2.0, -0.7, 0.0, 0.3, math.pi / 2, 2.9, math.pi], np.float32)


def _area(points, angle):
    E = len(points)
    xyt = np.zeros((E, 2, 3))
    xyt[:, 1, 0] = points[:, 0]
    xyt[:, 1, 1] = points[:, 1]
    xyt[:, 1, 2] = angle
    return O.pair_cost(xyt, grad=False)[0]


def test_rotation_angle_is_the_float32_path():
    for t in THETAS:
        a = MK.rotation_angle(t)
        assert abs(a - float(t)) < 1e-6
        assert a == float(np.float32(a))   # a float32 value, as the reference's NumPy makes it


def test_hulls_are_convex_and_ccw():
    for t in THETAS:
        for H in MK.forbidden_zone(t):
            assert 3 <= len(H) <= 8
            m = len(H)
            for k in range(m):
                assert MK._cross(H[k], H[(k + 1) % m], H[(k + 2) % m]) > 0.0


@pytest.mark.parametrize("theta", list(THETAS))
def test_outside_value_is_polygon_distance(theta):
    R = O.geometry()[3]
    rng = np.random.default_rng(7)
    pts = rng.uniform(-2.2 * R, 2.2 * R, size=(400, 2))
    val = MK.separation_distance(pts[:, 0], pts[:, 1], theta)
    out = val < -1e-6
    assert out.sum() > 100
    ang = MK.rotation_angle(theta)
    A = MK.tree_polygon()
    for (x, y), v in zip(pts[out], val[out]):
        d = MK.polygon_distance(A, MK.tree_polygon(x, y, ang))
        assert abs(-v - d) < 1e-12, (x, y, v, d)


@pytest.mark.parametrize("theta", list(THETAS))
def test_inside_test_matches_area_oracle(theta):
    R = O.geometry()[3]
    rng = np.random.default_rng(11)
    pts = rng.uniform(-1.6 * R, 1.6 * R, size=(3000, 2))
    val = MK.separation_distance(pts[:, 0], pts[:, 1], theta)
    area = _area(pts, MK.rotation_angle(theta))
    clear = np.abs(val) > 1e-5
    assert (val[clear] > 0).sum() > 200 and (val[clear] < 0).sum() > 200
    np.testing.assert_array_equal(val[clear] > 0, area[clear] > 1e-15)


def _exit_distance(p, dirs, angle, step=1e-3, rmax=2.5):
    """First distance along each ray from p at which the trees stop overlapping
    (area oracle), by marching then bisecting."""
    n = len(dirs)
    lo = np.zeros(n)
    hi = np.full(n, np.inf)
    r = step
    active = np.ones(n, bool)
    while active.any() and r < rmax:
        q = p[None, :] + r * dirs[active]
        free = _area(q, angle) <= 1e-15
        idx = np.nonzero(active)[0]
        hi[idx[free]] = r
        lo[idx[~free]] = r
        active[idx[free]] = False
        r += step
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        free = _area(p[None, :] + mid[:, None] * dirs, angle) <= 1e-15
        hi = np.where(free, mid, hi)
        lo = np.where(free, lo, mid)
    return hi


@pytest.mark.parametrize("theta", [np.float32(-2.0), np.float32(0.3), np.float32(math.pi)])
def test_inside_value_is_smallest_exit_distance(theta):
    R = O.geometry()[3]
    rng = np.random.default_rng(3)
    pts = rng.uniform(-1.2 * R, 1.2 * R, size=(400, 2))
    val = MK.separation_distance(pts[:, 0], pts[:, 1], theta)
    pick = np.nonzero((val > 0.01) & (val < 0.12))[0][:3]
    assert len(pick) == 3
    ang = MK.rotation_angle(theta)
    phi = np.linspace(0, 2 * math.pi, 1440, endpoint=False)
    dirs = np.stack([np.cos(phi), np.sin(phi)], 1)
    for i in pick:
        ex = _exit_distance(pts[i], dirs, ang)
        assert ex.min() >= val[i] - 1e-7, (pts[i], val[i], ex.min())
        assert ex.min() <= val[i] * (1 + 1e-3) + 1e-6, (pts[i], val[i], ex.min())
