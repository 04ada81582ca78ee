"""The GPU exact-separation table (pk_lut_build_exact_sep) against the FP64
oracle restatement of core/pack_minkowski.py, and the production table of
CollisionCostExactSeparation built from it."""
import math

import numpy as np
import pytest
import torch

from oracle import minkowski as MK

pytestmark = pytest.mark.gpu

THETAS = np.array([-math.pi, -2.0, -0.7, 0.0, 0.3, math.pi / 2, 2.9, math.pi], np.float32)


def _build(cuda, X, Y, T):
    from packing_b200 import _lib
    import ctypes
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(cuda)
    Yd = torch.from_numpy(np.ascontiguousarray(Y, np.float32)).to(cuda)
    Td = torch.from_numpy(np.ascontiguousarray(T, np.float32)).to(cuda)
    vals = torch.full((len(X), len(Y), len(T)), float("nan"), device=cuda)
    rc = _lib.load().pk_lut_build_exact_sep(_lib.ptr(Xd), len(X), _lib.ptr(Yd), len(Y), _lib.ptr(Td), len(T),
                                            _lib.ptr(vals), ctypes.c_void_p(_lib.stream_handle(None, cuda)))
    _lib.check(rc, "pk_lut_build_exact_sep")
    return vals.cpu().numpy()


def _compare(gpu, ora):
    assert np.isfinite(gpu).all()
    np.testing.assert_allclose(gpu, ora, rtol=0, atol=1e-6)
    # FP64 in the same operation order: equal but for the last bit of cos / sin
    assert (gpu == ora).mean() > 0.99
    clear = np.abs(ora) > 1e-6
    np.testing.assert_array_equal(gpu[clear] > 0, ora[clear] > 0)


def test_table_matches_oracle(cuda):
    from packing_b200.pack_cuda_lut import LookupTable
    X, Y, _ = LookupTable.default_grid(48, 48, 8)
    gpu = _build(cuda, X, Y, THETAS)
    _compare(gpu, MK.table(X, Y, THETAS))
    assert (gpu > 0).any() and (gpu < 0).any()


def test_batches_and_partial_tiles(cuda):
    """More slices than one batch of the builder; axes not multiples of its tiles."""
    X = np.linspace(-0.2, 1.1, 37, dtype=np.float32)
    Y = np.linspace(-1.15, 1.05, 53, dtype=np.float32)
    T = np.linspace(-np.pi, np.pi, 300, dtype=np.float32)
    gpu = _build(cuda, X, Y, T)
    pick = [0, 1, 255, 256, 299]
    _compare(gpu[:, :, pick], MK.table(X, Y, T[pick]))


def test_unsorted_axes(cuda):
    rng = np.random.default_rng(1)
    X = rng.uniform(-1.1, 1.1, 40).astype(np.float32)
    Y = rng.uniform(-1.1, 1.1, 33).astype(np.float32)
    T = rng.uniform(-np.pi, np.pi, 5).astype(np.float32)
    _compare(_build(cuda, X, Y, T), MK.table(X, Y, T))


def test_errors(cuda):
    from packing_b200 import _lib
    import ctypes
    L = _lib.load()
    x = torch.zeros(4, device=cuda)
    rc = L.pk_lut_build_exact_sep(_lib.ptr(x), 0, _lib.ptr(x), 4, _lib.ptr(x), 4, _lib.ptr(x), ctypes.c_void_p(0))
    assert rc != 0
    rc = L.pk_lut_build_exact_sep(None, 4, _lib.ptr(x), 4, _lib.ptr(x), 4, _lib.ptr(x), ctypes.c_void_p(0))
    assert rc != 0


def test_build_exact_separation_table(cuda):
    from packing_b200.pack_cuda_lut import LookupTable
    full = LookupTable.build_exact_separation(N_x=96, N_y=96, N_theta=72, trim_zeros=False, device=cuda)
    lut = LookupTable.build_exact_separation(N_x=96, N_y=96, N_theta=72, device=cuda)
    again = LookupTable.build_exact_separation(N_x=96, N_y=96, N_theta=72, device=cuda)
    assert lut.apply_quadratic_transform and full.apply_quadratic_transform
    assert torch.equal(lut.lut_d, again.lut_d)          # deterministic
    # the trim keeps the reference's rule: positive span plus one row / column on X and Y
    v = full.lut_d.cpu().numpy()
    X0, Y0, T0, v0 = LookupTable._trim_zero_edges(full.X, full.Y, full.theta, v, verbose=False)
    np.testing.assert_array_equal(lut.X, X0)
    np.testing.assert_array_equal(lut.Y, Y0)
    np.testing.assert_array_equal(lut.theta, T0)
    np.testing.assert_array_equal(lut.lut_d.cpu().numpy(), v0)
    assert lut.N_x < full.N_x and lut.N_y < full.N_y


def test_exact_table_cost_tracks_exact_separation(cuda):
    """The LUT cost of two trees (trilinear table, max(0, v)^2) follows the
    exact penetration depth at off-grid poses, to within the table's cell
    (about 0.007 in x and y, 0.0175 rad in theta)."""
    from packing_b200 import pack_cuda_lut
    from packing_b200.pack_cuda_lut import LookupTable
    lut = LookupTable.build_exact_separation(N_x=320, N_y=320, N_theta=360, device=cuda)
    rng = np.random.default_rng(5)
    E = 200
    xyt = np.zeros((E, 2, 3), np.float32)
    xyt[:, 1, 0] = rng.uniform(-0.6, 0.6, E)
    xyt[:, 1, 1] = rng.uniform(-0.8, 0.8, E)
    xyt[:, 1, 2] = rng.uniform(-3.0, 3.0, E)
    c = torch.empty(E, device=cuda)
    pack_cuda_lut.overlap_multi_ensemble(torch.from_numpy(xyt).to(cuda), c, lut)
    exact = np.array([max(0.0, float(MK.separation_distance([x], [y], t)[0])) for x, y, t in xyt[:, 1, :]])
    got = np.sqrt(c.cpu().numpy())
    assert (exact > 0.03).sum() > 50
    err = np.abs(got - exact)
    assert err.max() < 8e-3, err.max()
    assert np.median(err[exact > 0]) < 1e-3


def test_forbidden_zone_has_no_holes(cuda):
    """Shapely measures a single polygon to its exterior ring and the builder to
    the whole union boundary; they agree when Z has no hole.  On a full-plane
    grid every connected region of non-overlapping poses reaches the grid's
    edge, for every slice."""
    from scipy import ndimage
    from packing_b200.pack_cuda_lut import tree_max_radius
    R = tree_max_radius()
    X = np.linspace(-2.05 * R, 2.05 * R, 401, dtype=np.float32)
    T = np.linspace(-np.pi, np.pi, 181, dtype=np.float32)
    vals = _build(cuda, X, X, T)
    for k in range(len(T)):
        lab, n = ndimage.label(vals[:, :, k] < 0)
        edge = set(np.unique(np.concatenate([lab[0], lab[-1], lab[:, 0], lab[:, -1]]))) - {0}
        assert set(range(1, n + 1)) == edge, (k, float(T[k]), n, sorted(edge))


def test_single_point_and_single_slice_grids(cuda):
    """Grids of one point and of one slice (too few values for the share of
    bit-identical entries to mean anything: tolerance and sign only)."""
    T = np.array([0.7], np.float32)
    for X, Y in ((np.array([0.1], np.float32), np.array([-0.05], np.float32)),
                 (np.linspace(-0.3, 1.0, 9, dtype=np.float32),) * 2):
        gpu, ora = _build(cuda, X, Y, T), MK.table(X, Y, T)
        np.testing.assert_allclose(gpu, ora, rtol=0, atol=1e-6)
        clear = np.abs(ora) > 1e-6
        np.testing.assert_array_equal(gpu[clear] > 0, ora[clear] > 0)
