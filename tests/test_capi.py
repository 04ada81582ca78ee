"""The C-ABI library: builds, loads, exports every symbol include/packb200.h
declares, and its geometry tables match the oracle's (CPU only)."""
import ctypes
import os
import re

import numpy as np

from oracle import oracle as O
from packing_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "packb200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(pk_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)


def test_default_geometry_matches_oracle():
    g = _lib.default_geometry()
    pxy, pnv, txy, R, cut, area = O.geometry()
    assert g.n_tree_verts == 15
    assert list(g.piece_nv) == list(pnv)
    tree = np.array([[g.tree_xy[i][0], g.tree_xy[i][1]] for i in range(15)])
    np.testing.assert_allclose(tree, txy, rtol=0, atol=1e-15)
    assert abs(g.max_radius - R) < 1e-15
    assert abs(g.area - area) < 1e-15
    # pieces as given (before orientation): same vertex sets as the oracle's CCW pieces
    for p in range(4):
        a = {(round(g.piece_xy[p][v][0], 12), round(g.piece_xy[p][v][1], 12)) for v in range(pnv[p])}
        b = {(round(pxy[p, v, 0], 12), round(pxy[p, v, 1], 12)) for v in range(pnv[p])}
        assert a == b


def test_errors_are_codes_not_crashes():
    L = _lib.load()
    # no device on this host: the call reports an error instead of crashing
    spec = _lib.PkCostSpec()
    rc = L.pk_cost(None, None, 1, 4, None, ctypes.byref(spec), None, None, None, None)
    assert rc != 0
    assert isinstance(L.pk_last_error(), bytes) and len(L.pk_last_error()) > 0
    rc = L.pk_lap_solve(None, 1, 300, None, None, None, None)
    assert rc == -4
    assert b"256" in L.pk_last_error()
    assert L.pk_relax_workspace_floats(None, 10, 200, 10) == 2 * 10 * 10 * 603


def test_probes_reject_bad_arguments_before_launching():
    """The roofline probes validate their arguments on the host and return a
    status (no launch, so this runs without a device)."""
    L = _lib.load()
    assert L.pk_gather_probe(None, 256, 256, 360, None, 1, 1, 1, 0, None) != 0
    assert b"pk_gather_probe" in L.pk_last_error()
    assert L.pk_fma_probe(None, 1, 1, 1, None) != 0
    assert b"pk_fma_probe" in L.pk_last_error()


def test_diversity_entry_points_check_arguments_on_the_host():
    """NULL arrays and a (pop, ref) pair count beyond the one-CTA-per-pair
    grid are refused with a status before any launch (no device needed)."""
    L = _lib.load()
    for fn in ("pk_diversity_costs", "pk_diversity_matrix"):
        assert getattr(L, fn)(None, None, 2, 3, 10, 1, None, None) == -1, fn
        assert b"NULL" in L.pk_last_error()
        assert getattr(L, fn)(None, None, 70000, 70000, 10, 1, None, None) == -4, fn
        assert b"grid limit" in L.pk_last_error()
    assert L.pk_diversity_shortcut(None, None, 2, 3, 10, 1.0, 0.0, 0, None, None) == -1
    assert L.pk_diversity_shortcut(None, None, 70000, 70000, 10, 1.0, 0.0, 0, None, None) == -4
    assert L.pk_diversity_costs(None, None, -1, 3, 10, 1, None, None) == -1
    assert L.pk_diversity_costs(None, None, 0, 3, 10, 1, None, None) == 0     # nothing to do


def test_allocation_free_relaxation_needs_init_first():
    """pk_relax_noalloc checks pk_init before any CUDA call: on a host where
    pk_init has not run it returns PK_ENOTINIT."""
    L = _lib.load()
    prm = _lib.PkRelaxParams()
    prm.history = 10
    assert L.pk_relax_noalloc(None, None, 1, 10, None, ctypes.byref(prm), None, None, None, None, None) != 0
