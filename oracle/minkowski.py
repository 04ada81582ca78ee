"""FP64 CPU restatement of ``core/pack_minkowski.py`` -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module; the product never does.

The reference tabulates, for the production collision term of the GA
(``CollisionCostExactSeparation``, ``pack_cost.py:1119-1215``), the signed
separation of tree 1 (origin, unrotated) and tree 2 (at ``t = (dx, dy)``,
rotated by theta) with shapely (``separation_distance``,
``pack_minkowski.py:210-266``):

* the forbidden zone Z is the union over the 4 x 4 convex piece pairs of the
  Minkowski difference ``hull{a - b}`` (``:34-62``, ``:103-137``);
* the value is ``+dist(t, boundary)`` when Z contains t strictly and
  ``-dist(t, boundary)`` otherwise (``:253-264``).

Shapely is not available here, so the union is restated directly: the 16
hulls by Andrew's monotone chain, and the boundary of their union as every
hull edge minus its parts strictly inside another hull.  Shapely measures a
single polygon to its exterior ring; this restatement measures to the whole
union boundary (they differ only where Z has a hole).

Arithmetic: Python floats (FP64, no fused multiply-add), every operation in
the order the GPU builder uses, so the two agree up to the last-bit
difference of the platforms' cos and sin.  The rotation angle follows the
reference's float32 path: ``np.degrees`` of a float32 theta and shapely's
``angle * pi / 180`` evaluated by NumPy in float32.

Pinning: no golden values for this path exist in the reference's tests, and
shapely cannot run here, so parity with the reference is UNPINNED.  The
tests check this restatement against two independent facts instead: outside
Z the value is minus the polygon distance of the two trees, and the inside
test agrees with the overlap-area oracle.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as _oracle


def rotation_angle(theta) -> float:
    """The angle (radians, FP64) by which the reference turns tree 2 for the
    float32 table angle ``theta``: ``affinity.rotate(p, np.degrees(theta))``
    (``pack_minkowski.py:82-83``) with shapely's ``angle * pi / 180.0``."""
    deg = np.degrees(np.float32(theta))
    rad = np.float32(np.float32(deg * np.float32(math.pi)) / np.float32(180.0))
    return float(rad)


def _cross(o, a, b):
    return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])


def convex_hull(points):
    """CCW hull without collinear points (Andrew's monotone chain)."""
    pts = sorted(points)
    if len(pts) <= 2:
        return pts
    lower, upper = [], []
    for p in pts:
        while len(lower) >= 2 and _cross(lower[-2], lower[-1], p) <= 0.0:
            lower.pop()
        lower.append(p)
    for p in reversed(pts):
        while len(upper) >= 2 and _cross(upper[-2], upper[-1], p) <= 0.0:
            upper.pop()
        upper.append(p)
    return lower[:-1] + upper[:-1]


def _pieces():
    pxy, pnv, _, _, _, _ = _oracle.geometry()
    return [[(float(pxy[p, v, 0]), float(pxy[p, v, 1])) for v in range(int(pnv[p]))] for p in range(4)]


def forbidden_zone(theta):
    """The 16 convex Minkowski differences (CCW vertex lists) for the table
    angle theta, tree 1's piece p against tree 2's piece q at index 4 p + q."""
    ang = rotation_angle(theta)
    cs, sn = math.cos(ang), math.sin(ang)
    pieces = _pieces()
    hulls = []
    for P in pieces:
        for Q in pieces:
            pts = []
            for (ax, ay) in P:
                for (qx, qy) in Q:
                    bx = cs * qx - sn * qy
                    by = sn * qx + cs * qy
                    pts.append((ax - bx, ay - by))
            hulls.append(convex_hull(pts))
    return hulls


def union_boundary(hulls):
    """Segments (S, 4) of the boundary of the union: every hull edge minus
    the parts strictly inside another hull."""
    segs = []
    for r, H in enumerate(hulls):
        m = len(H)
        for k in range(m):
            a, b = H[k], H[(k + 1) % m]
            iv = []
            for o, G in enumerate(hulls):
                if o == r or len(G) < 3:
                    continue
                lo, hi, empty = 0.0, 1.0, False
                for j in range(len(G)):
                    u, w = G[j], G[(j + 1) % len(G)]
                    f0, f1 = _cross(u, w, a), _cross(u, w, b)
                    if f0 <= 0.0 and f1 <= 0.0:
                        empty = True
                    elif f0 > 0.0 and f1 <= 0.0:
                        hi = min(hi, f0 / (f0 - f1))
                    elif f0 <= 0.0 and f1 > 0.0:
                        lo = max(lo, f0 / (f0 - f1))
                    if lo >= hi:
                        empty = True
                    if empty:
                        break
                if not empty:
                    iv.append((lo, hi))
            iv.sort(key=lambda x: x[0])
            dx, dy = b[0] - a[0], b[1] - a[1]
            cur = 0.0
            for i in range(len(iv) + 1):
                nxt = iv[i][0] if i < len(iv) else 1.0
                if nxt > cur:
                    segs.append((a[0] if cur == 0.0 else a[0] + cur * dx, a[1] if cur == 0.0 else a[1] + cur * dy,
                                 b[0] if nxt == 1.0 else a[0] + nxt * dx, b[1] if nxt == 1.0 else a[1] + nxt * dy))
                if i < len(iv):
                    cur = max(cur, iv[i][1])
    return np.array(segs, dtype=np.float64).reshape(-1, 4)


def inside(hulls, dx, dy):
    """Strict containment of the points (dx, dy) in the union."""
    dx = np.asarray(dx, np.float64)
    dy = np.asarray(dy, np.float64)
    res = np.zeros(dx.shape, bool)
    for H in hulls:
        if len(H) < 3:
            continue
        ok = np.ones(dx.shape, bool)
        m = len(H)
        for j in range(m):
            o, a = H[j], H[(j + 1) % m]
            ok &= (a[0] - o[0]) * (dy - o[1]) - (a[1] - o[1]) * (dx - o[0]) > 0.0
        res |= ok
    return res


def segment_distance(segs, dx, dy):
    """Smallest distance from each point to the segments, FP64 in the order
    of the GPU builder."""
    dx = np.asarray(dx, np.float64).reshape(-1, 1)
    dy = np.asarray(dy, np.float64).reshape(-1, 1)
    ax, ay, bx, by = (segs[:, i][None, :] for i in range(4))
    ex, ey = bx - ax, by - ay
    px, py = dx - ax, dy - ay
    ll = ex * ex + ey * ey
    pe = px * ex + py * ey
    with np.errstate(divide="ignore", invalid="ignore"):
        u = np.where(ll > 0.0, pe / np.where(ll > 0.0, ll, 1.0), 0.0)
    u = np.clip(u, 0.0, 1.0)
    qx, qy = px - u * ex, py - u * ey
    return np.sqrt(np.min(qx * qx + qy * qy, axis=1))


def separation_distance(dx, dy, theta):
    """Signed separation (FP64) of the points for the table angle theta."""
    hulls = forbidden_zone(theta)
    segs = union_boundary(hulls)
    dx = np.asarray(dx, np.float64).ravel()
    dy = np.asarray(dy, np.float64).ravel()
    d = segment_distance(segs, dx, dy)
    return np.where(inside(hulls, dx, dy), d, -d)


def table(X, Y, theta):
    """vals[ix, iy, it] float32 over the grid, like the GPU builder."""
    X = np.asarray(X, np.float32)
    Y = np.asarray(Y, np.float32)
    theta = np.asarray(theta, np.float32)
    gx, gy = np.meshgrid(X.astype(np.float64), Y.astype(np.float64), indexing="ij")
    out = np.zeros((len(X), len(Y), len(theta)), np.float32)
    for k, t in enumerate(theta):
        out[:, :, k] = separation_distance(gx.ravel(), gy.ravel(), t).reshape(len(X), len(Y)).astype(np.float32)
    return out


def polygon_distance(A, B):
    """Distance between two disjoint simple polygons (vertex arrays): the
    smallest vertex-to-edge distance either way."""
    def vert_to_edges(V, W):
        a = W
        b = np.roll(W, -1, axis=0)
        segs = np.concatenate([a, b], axis=1)
        return segment_distance(segs, V[:, 0], V[:, 1]).min()
    return min(vert_to_edges(A, B), vert_to_edges(B, A))


def tree_polygon(x=0.0, y=0.0, angle=0.0):
    """The oracle's 15-vertex tree turned by angle (radians) and moved to (x, y)."""
    _, _, txy, _, _, _ = _oracle.geometry()
    c, s = math.cos(angle), math.sin(angle)
    return np.stack([c * txy[:, 0] - s * txy[:, 1] + x, s * txy[:, 0] + c * txy[:, 1] + y], axis=1)
