"""CPU restatement of the GA moves (core/pack_move.py) -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module; the product never does.

The reference applies its moves with cupy on whole batches and draws from a
cupy generator.  This restatement applies them one row at a time, in numpy,
with the reference's dtypes (float64 draws, float32 poses and float32
operations where the reference combines float32 arrays with Python
scalars), and takes its draws from the same Philox4x32-10 stream as the
GPU kernels, so a row's result can be compared bit for bit.

Philox4x32-10 is restated from Salmon, Moraes, Dror and Shaw, "Parallel
random numbers: as easy as 1, 2, 3" (SC 2011) and pinned to three of
Random123's known-answer vectors in ``tests/test_moves_oracle.py``.

Draw k of a row: counter (k // 2, row position, call low word, call high
word), key (seed low word, seed high word); the 128-bit block gives two
uniforms, (x0 >> 5, x1 >> 6) and (x2 >> 5, x3 >> 6) as 53-bit fractions.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32
M32 = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    c = [int(v) & M32 for v in ctr]
    k0, k1 = int(key[0]) & M32, int(key[1]) & M32
    for _ in range(10):
        p0 = 0xD2511F53 * c[0]
        p1 = 0xCD9E8D57 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & M32, p1 & M32, ((p0 >> 32) ^ c[3] ^ k1) & M32, p0 & M32]
        k0 = (k0 + 0x9E3779B9) & M32
        k1 = (k1 + 0xBB67AE85) & M32
    return c


class Stream:
    """The draws of one row: ``u()`` takes the next one."""

    def __init__(self, seed: int, call: int, row: int):
        self.key = (seed & M32, (seed >> 32) & M32)
        self.ctr = (row & M32, call & M32, (call >> 32) & M32)
        self.next = 0

    def draw(self, k: int) -> float:
        x = philox4x32_10((k >> 1, self.ctr[0], self.ctr[1], self.ctr[2]), self.key)
        a, b = (x[2], x[3]) if k & 1 else (x[0], x[1])
        return ((a >> 5) * 67108864.0 + (b >> 6)) * (1.0 / 9007199254740992.0)

    def u(self) -> float:
        v = self.draw(self.next)
        self.next += 1
        return v

    def uniform(self, lo, hi) -> float:
        lo, hi = float(lo), float(hi)
        return lo + (hi - lo) * self.u()

    def integers(self, lo: int, hi_excl: int) -> int:
        span = hi_excl - lo
        k = int(math.floor(self.u() * span))
        return lo + min(max(k, 0), span - 1)


def pymod(a, b):
    """numpy's remainder of float64 / float32 scalars (sign of the divisor)."""
    return type(a)(np.remainder(a, b))


# ---- edge spacers and move centres (kaggle_support.py) -------------------

def spacer_ok(geno, x, y, h0):
    """EdgeSpacerBasic._check_valid (kaggle_support.py:497-513) for one
    location, float32; EdgeSpacerDummy accepts everything."""
    sp = geno["spacer"]
    if sp is None:
        return True
    x, y, h0 = F(x), F(y), F(h0)
    mg = F(geno["margin"])
    half = h0 / F(2)
    if abs(x) >= half - F(sp["dist_x"]) - mg or abs(y) >= half - F(sp["dist_y"]) - mg:
        return True
    hs = half - mg
    dc = F(sp["dist_corner"])
    d = [abs(x - hs) + abs(y - hs), abs(x + hs) + abs(y - hs), abs(x - hs) + abs(y + hs), abs(x + hs) + abs(y + hs)]
    return any(v <= dc for v in d)


def move_centers(geno, filt, ec, h, s: Stream):
    """generate_move_centers of the population's class for one row; ec None
    means no edge clearance.  Square: kaggle_support.py:881-1030;
    Symmetric90: :1211-1268; Symmetric180: :1409-1620."""
    h0, h1, h2 = F(h[0]), F(h[1]), F(h[2])
    kind = geno["kind"]
    sp = geno["spacer"]
    analytic = sp is not None and sp["dist_corner"] == 0.0 and filt
    if kind == "square":
        if ec is not None:
            size = F(float(h0) - ec * 2)
            hs = float(size / F(2))
            return F(F(s.uniform(-hs, hs)) + h1), F(F(s.uniform(-hs, hs)) + h2)
        if analytic:
            size = h0
            half = size / F(2)
            mg = F(geno["margin"])
            xt = half - F(sp["dist_x"]) - mg
            yt = half - F(sp["dist_y"]) - mg
            area_A = (half - xt) * size
            area_B = area_A
            area_C = (F(2) * xt) * (half - yt)
            area_D = area_C
            total = max(area_A + area_B + area_C + area_D, F(1e-10))
            pA, pAB, pABC = area_A / total, (area_A + area_B) / total, (area_A + area_B + area_C) / total
            sel = s.u()
            if sel < float(pA):
                x, y = s.uniform(-half, -xt), s.uniform(-half, half)
            elif sel < float(pAB):
                x, y = s.uniform(xt, half), s.uniform(-half, half)
            elif sel < float(pABC):
                x, y = s.uniform(-xt, xt), s.uniform(yt, half)
            else:
                x, y = s.uniform(-xt, xt), s.uniform(-half, -yt)
            return F(F(x) + h1), F(F(y) + h2)
        hs = float(h0 / F(2))
        while True:
            x = F(F(s.uniform(-hs, hs)) + h1)
            y = F(F(s.uniform(-hs, hs)) + h2)
            if not filt or spacer_ok(geno, x, y, h0):
                return x, y
    if kind == "sym90":
        assert not filt
        e = 0.0 if ec is None else ec
        size = h0 if ec is None else F(float(h0) - ec * 2)
        assert float(h0) >= 4 * e
        lo = -float(size / F(2))
        while True:
            x, y = s.uniform(lo, 0.0), s.uniform(lo, 0.0)
            if x + y <= -2 * e:
                return F(x + float(h1)), F(y + float(h2))
    # sym180
    if ec is not None:
        size = F(float(h0) - ec * 2)
        half = size / F(2)
        assert float(h0) >= 4 * ec
        H = float(half)
        area_A = (H - ec) * float(size)
        area_B = ec * (H - ec)
        area_C = ec * (H - ec)
        total = area_A + area_B + area_C
        pA, pAB = area_A / total, (area_A + area_B) / total
        sel = s.u()
        if sel < pA:
            x, y = s.uniform(-H, -ec), s.uniform(-H, H)
        elif sel < pAB:
            x, y = s.uniform(-ec, 0.0), s.uniform(ec, H)
        else:
            x, y = s.uniform(-ec, 0.0), s.uniform(-H, -ec)
        return F(F(x) + h1), F(F(y) + h2)
    if analytic:
        size = h0
        half = size / F(2)
        mg = F(geno["margin"])
        xt = half - F(sp["dist_x"]) - mg
        yt = half - F(sp["dist_y"]) - mg
        area_A = (half - xt) * size
        area_B = xt * (half - yt)
        area_C = xt * (half - yt)
        total = max(area_A + area_B + area_C, F(1e-10))
        pA, pAB = area_A / total, (area_A + area_B) / total
        sel = s.u()
        if sel < float(pA):
            x, y = s.uniform(-half, -xt), s.uniform(-half, half)
        elif sel < float(pAB):
            x, y = s.uniform(-xt, 0.0), s.uniform(yt, half)
        else:
            x, y = s.uniform(-xt, 0.0), s.uniform(-half, -yt)
        return F(F(x) + h1), F(F(y) + h2)
    hs = float(h0 / F(2))
    while True:
        x, y = s.uniform(-hs, 0.0), s.uniform(-hs, hs)
        fx, fy = F(x + float(h1)), F(y + float(h2))
        if not filt or spacer_ok(geno, fx, fy, h0):
            return fx, fy


def sample_tree(geno, filt, xyt, h0, s: Stream):
    """_sample_trees_to_mutate (pack_move.py:58-116) for one row."""
    n = xyt.shape[0]
    if not filt:
        return s.integers(0, n)
    valid = np.array([spacer_ok(geno, xyt[i, 0], xyt[i, 1], h0) for i in range(n)])
    if not valid.any():
        valid[:] = True
    r = int(s.u() * int(valid.sum()))
    return int(np.argmax(np.cumsum(valid) >= r + 1))


def canonicalize(kind, xyt):
    """canonicalize_xyt of the mate's class (kaggle_support.py:1053-1088, 1287-1310), float32."""
    x, y, t = xyt[:, 0].copy(), xyt[:, 1].copy(), xyt[:, 2].copy()
    if kind == "sym90":
        q1 = (x > 0) & (y > 0)
        q2 = (x <= 0) & (y > 0)
        q4 = (x > 0) & (y <= 0)
        nx = np.where(q1, -x, x)
        nx = np.where(q2, -y, nx)
        nx = np.where(q4, y, nx)
        ny = np.where(q1, -y, y)
        ny = np.where(q2, x, ny)
        ny = np.where(q4, -x, ny)
        nt = np.where(q1, t + F(np.pi), t)
        nt = np.where(q2, t + F(np.pi / 2), nt)
        nt = np.where(q4, t + F(3 * np.pi / 2), nt)
    elif kind == "sym180":
        r = x > 0
        nx, ny = np.where(r, -x, x), np.where(r, -y, y)
        nt = np.where(r, t + F(np.pi), t)
    else:
        return xyt
    out = np.stack([nx, ny, np.remainder(nt.astype(F), F(2 * np.pi))], 1).astype(F)
    return out


def _argsort(d):
    return np.argsort(d, kind="stable")


def _linf(px, py, cx, cy):
    return np.maximum(np.abs(px - cx), np.abs(py - cy))


# ---- the moves, one row ---------------------------------------------------

def move_random_tree(mv, geno, filt, xyt, h, s):   # pack_move.py:161-188
    t = sample_tree(geno, filt, xyt, h[0], s)
    cx, cy = move_centers(geno, filt, None, h, s)
    th = s.uniform(-np.pi, np.pi)
    xyt[t] = [cx, cy, F(th)]


def jiggle_tree(mv, geno, filt, xyt, h, s):   # pack_move.py:191-224
    t = sample_tree(geno, filt, xyt, h[0], s)
    off = [s.uniform(-mv["max_xy_move"], mv["max_xy_move"]), s.uniform(-mv["max_xy_move"], mv["max_xy_move"]),
           s.uniform(-mv["max_theta_move"], mv["max_theta_move"])]
    for k in range(3):
        xyt[t, k] = F(float(xyt[t, k]) + off[k])


def jiggle_cluster(mv, geno, filt, xyt, h, s):   # pack_move.py:227-298
    n = xyt.shape[0]
    cx, cy = move_centers(geno, filt, None, h, s)
    maxj, minj = min(mv["max_N_trees"], n), min(mv["min_N_trees"], n)
    nj = s.integers(minj, maxj + 1)
    base = s.next
    s.next += 3 * maxj
    mxy, mth = mv["max_xy_move"], mv["max_theta_move"]
    ox = [-mxy + (mxy - (-mxy)) * s.draw(base + j) for j in range(maxj)]
    oy = [-mxy + (mxy - (-mxy)) * s.draw(base + maxj + j) for j in range(maxj)]
    ot = [-mth + (mth - (-mth)) * s.draw(base + 2 * maxj + j) for j in range(maxj)]
    dx = xyt[:, 0] - cx
    dy = xyt[:, 1] - cy
    d = dx * dx + dy * dy
    order = _argsort(d)[:maxj]
    for j, t in enumerate(order):
        mask = 1.0 if j < nj else 0.0
        xyt[t, 0] = F(float(xyt[t, 0]) + ox[j] * mask)
        xyt[t, 1] = F(float(xyt[t, 1]) + oy[j] * mask)
        xyt[t, 2] = F(float(xyt[t, 2]) + ot[j] * mask)


def translate(mv, geno, filt, xyt, h, s):   # pack_move.py:301-333
    h0 = F(h[0])
    hs = float(h0 / F(2))
    ox, oy = s.uniform(-hs, hs), s.uniform(-hs, hs)
    for i in range(xyt.shape[0]):
        xyt[i, 0] = F(pymod(float(xyt[i, 0]) + ox, float(h0)) - hs)
        xyt[i, 1] = F(pymod(float(xyt[i, 1]) + oy, float(h0)) - hs)


def twist(mv, geno, filt, xyt, h, s):   # pack_move.py:336-382
    cx, cy = move_centers(geno, filt, None, h, s)
    a = s.uniform(-np.pi, np.pi)
    r = s.uniform(mv["min_radius"], mv["max_radius"])
    for i in range(xyt.shape[0]):
        dx, dy = xyt[i, 0] - cx, xyt[i, 1] - cy
        dist = np.sqrt(dx * dx + dy * dy)
        tw = a * max(0.0, 1.0 - float(dist) / r)
        c, sn = math.cos(tw), math.sin(tw)
        xyt[i, 0] = F(float(cx) + float(dx) * c - float(dy) * sn)
        xyt[i, 1] = F(float(cy) + float(dx) * sn + float(dy) * c)
        xyt[i, 2] = F(float(xyt[i, 2]) + tw)


def crossover(mv, geno, filt, xyt, h, mate_xyt, mate_h, s):   # pack_move.py:406-632
    n = xyt.shape[0]
    min_t = min(mv["min_N_trees"], n)
    max_t = min(int(np.round(mv["max_N_trees_ratio"] * n)), n)
    if max_t < min_t:
        max_t = min_t
    nrep = s.integers(min_t, max_t + 1)
    rot = s.integers(0, 4)
    mirror = s.integers(0, 2) == 1
    if mv["simple_mate_location"]:
        NT = n * {"square": 1, "sym90": 4, "sym180": 2}[geno["kind"]]
        ss = float(F(h[0])) * math.sqrt(nrep / NT)
        icx, icy = move_centers(geno, filt, ss / 2, h, s)
        mcx, mcy = move_centers(geno, filt, ss / 2, h, s)
        dm = _linf(mate_xyt[:, 0], mate_xyt[:, 1], mcx, mcy)
    else:
        icx, icy = move_centers(geno, filt, None, h, s)
        sgx, sgy = s.integers(0, 2) * 2 - 1, s.integers(0, 2) * 2 - 1
        ratio = F(mate_h[0]) / F(h[0])
        mcx = float(abs(icx - F(h[1])) * ratio) * sgx + float(F(mate_h[1]))
        mcy = float(abs(icy - F(h[2])) * ratio) * sgy + float(F(mate_h[2]))
        dm = np.maximum(np.abs(mate_xyt[:, 0].astype(np.float64) - mcx), np.abs(mate_xyt[:, 1].astype(np.float64) - mcy))
    di = _linf(xyt[:, 0], xyt[:, 1], icx, icy)
    ind = _argsort(di)[:nrep]
    mat = _argsort(dm)[:nrep]
    # centres of mass of the selections (float32 sums in rank order)
    sums = [F(0)] * 4
    for a, b in zip(ind, mat):
        sums = [sums[0] + xyt[a, 0], sums[1] + xyt[a, 1], sums[2] + mate_xyt[b, 0], sums[3] + mate_xyt[b, 1]]
    icm = [float(sums[0]) / nrep, float(sums[1]) / nrep]
    mcm = [float(sums[2]) / nrep, float(sums[3]) / nrep]
    ang = rot * (np.pi / 2)
    c, sn = math.cos(ang), math.sin(ang)
    new = []
    for b in mat:
        dx, dy = float(mate_xyt[b, 0]) - mcm[0], float(mate_xyt[b, 1]) - mcm[1]
        th = mate_xyt[b, 2]
        if mirror:
            dy = -dy
            th = F(np.pi) - th
        th = float(th)
        if rot != 0:
            dx, dy = dx * c - dy * sn, dx * sn + dy * c
            th = th + ang
        new.append([F(icm[0] + dx), F(icm[1] + dy), F(th)])
    for a, v in zip(ind, new):
        xyt[a] = v


def crossover2(mv, geno, filt, xyt, h, mate_xyt, mate_h, mate_kind, s):   # pack_move.py:635-1033
    n = xyt.shape[0]
    rot = s.integers(0, 4) if mv["do_90_rotation"] else 2 * s.integers(0, 2)
    mirror = s.integers(0, 2) == 1
    # _apply_orientation_preselection (:1003-1033)
    mate = mate_xyt.copy()
    x, y, t = mate[:, 0].copy(), mate[:, 1].copy(), mate[:, 2].copy()
    if mirror:
        y = -y
        t = F(np.pi) - t
    ang = rot * (np.pi / 2)
    c, sn = math.cos(ang), math.sin(ang)
    if rot != 0:
        rx = x.astype(np.float64) * c - y.astype(np.float64) * sn
        ry = x.astype(np.float64) * sn + y.astype(np.float64) * c
        t = (t.astype(np.float64) + ang).astype(F)
        x, y = rx.astype(F), ry.astype(F)
    mate = canonicalize(mate_kind, np.stack([x, y, t], 1).astype(F))
    if filt:
        vi = np.array([spacer_ok(geno, xyt[i, 0], xyt[i, 1], h[0]) for i in range(n)])
        vm = np.array([spacer_ok(geno, mate[i, 0], mate[i, 1], mate_h[0]) for i in range(n)])
    else:
        vi = vm = np.ones(n, bool)
    usable = max(min(int(vi.sum()), int(vm.sum())), 0)
    min_a = min(min(mv["min_N_trees"], n), usable)
    max_a = min(int(math.floor(mv["max_N_trees_ratio"] * usable)), usable)
    max_a = max(max_a, min_a)
    nrep = min_a + int(math.floor(s.u() * (max_a - min_a + 1)))
    if not mv["decouple_mate_location"]:
        lx, ly = move_centers(geno, filt, None, h, s)
        mlx, mly = lx - F(h[1]) + F(mate_h[1]), ly - F(h[2]) + F(mate_h[2])
    elif mv["use_edge_clearance_when_decoupled"]:
        NT = n * {"square": 1, "sym90": 4, "sym180": 2}[mate_kind]
        ss = float(F(h[0])) * math.sqrt(nrep / NT)
        lx, ly = move_centers(geno, filt, ss / 2, h, s)
        mlx, mly = move_centers(geno, filt, ss / 2, h, s)
    else:
        lx, ly = move_centers(geno, filt, None, h, s)
        mlx, mly = move_centers(geno, filt, None, h, s)
    df = mv["distance_function"]
    px, py, qx, qy = xyt[:, 0], xyt[:, 1], mate[:, 0], mate[:, 1]
    if df == "stripe":
        la = s.uniform(0, 2 * np.pi)
        nx, ny = -math.sin(la), math.cos(la)
        di = np.abs((px - lx).astype(np.float64) * nx + (py - ly).astype(np.float64) * ny)
        dm = np.abs((qx - mlx).astype(np.float64) * nx + (qy - mly).astype(np.float64) * ny)
    elif df == "square":
        di = _linf(px, py, lx, ly)
        dm = _linf(qx, qy, mlx, mly)
    elif df == "square90":
        di = np.minimum(np.minimum(_linf(px, py, lx, ly), _linf(-py, px, lx, ly)),
                        np.minimum(_linf(-px, -py, lx, ly), _linf(py, -px, lx, ly)))
        ds = np.stack([_linf(qx, qy, mlx, mly), _linf(-qy, qx, mlx, mly), _linf(-qx, -qy, mlx, mly),
                       _linf(qy, -qx, mlx, mly)], 1)
        dm = np.minimum(np.minimum(ds[:, 0], ds[:, 1]), np.minimum(ds[:, 2], ds[:, 3]))
        k = np.argmin(ds, axis=1)
        tx = np.select([k == 0, k == 1, k == 2, k == 3], [qx, -qy, -qx, qy])
        ty = np.select([k == 0, k == 1, k == 2, k == 3], [qy, qx, -qy, -qx])
        tt = np.select([k == 0, k == 1, k == 2, k == 3],
                       [mate[:, 2], mate[:, 2] + F(np.pi / 2), mate[:, 2] + F(np.pi), mate[:, 2] + F(3 * np.pi / 2)])
        mate = np.stack([tx, ty, tt], 1).astype(F)
    elif df == "square180":
        di = np.minimum(_linf(px, py, lx, ly), _linf(-px, -py, lx, ly))
        d0, d1 = _linf(qx, qy, mlx, mly), _linf(-qx, -qy, mlx, mly)
        dm = np.minimum(d0, d1)
        k = np.argmin(np.stack([d0, d1], 1), axis=1)
        mate = np.stack([np.where(k == 1, -qx, qx), np.where(k == 1, -qy, qy),
                         np.where(k == 1, mate[:, 2] + F(np.pi), mate[:, 2])], 1).astype(F)
    else:
        raise ValueError(df)
    di = np.where(vi, di.astype(np.float64), np.inf)
    dm = np.where(vm, dm.astype(np.float64), np.inf)
    ind = _argsort(di)[:nrep]
    mat = _argsort(dm)[:nrep]
    new = mate[mat].copy()
    if mv["decouple_mate_location"]:
        new[:, 0] += lx - mlx
        new[:, 1] += ly - mly
    xyt[ind] = new


MOVES = {"MoveRandomTree": move_random_tree, "JiggleRandomTree": jiggle_tree, "JiggleCluster": jiggle_cluster,
         "Translate": translate, "Twist": twist}


def apply(entries, geno, xyt, h, inds_to_do, mate_xyt, mate_h, inds_mate, seed, call, mate_kind=None):
    """MoveSelector.do_move_vec restated per row: entries [(name, params, weight)];
    returns (new xyt, chosen entry per row)."""
    xyt = np.array(xyt, dtype=F, copy=True)
    w = np.array([e[2] for e in entries], dtype=np.float64)
    cum = np.cumsum((w / w.sum()).astype(F), dtype=F)
    mate_kind = mate_kind or geno["kind"]
    chosen = []
    for pos, row in enumerate(inds_to_do):
        s = Stream(seed, call, pos)
        m = int(np.searchsorted(cum.astype(np.float64), s.u(), side="left"))
        if m >= len(entries):
            chosen.append(-1)
            continue
        chosen.append(m)
        name, mv, _ = entries[m]
        filt = geno["filter"] and mv.get("respect_edge_spacer_filter", True)
        X = xyt[row]
        if name in MOVES:
            MOVES[name](mv, geno, filt, X, h[row], s)
        elif name == "Crossover":
            crossover(mv, geno, filt, X, h[row], mate_xyt[inds_mate[pos]], mate_h[inds_mate[pos]], s)
        elif name == "Crossover2":
            crossover2(mv, geno, filt, X, h[row], mate_xyt[inds_mate[pos]], mate_h[inds_mate[pos]], mate_kind, s)
        else:
            raise ValueError(name)
        xyt[row] = X
    return xyt, np.array(chosen)
