"""Drop-in for ``core/pack_cuda.py``: batched overlap / separation and
boundary-distance cost with analytic gradients, on sm_100a.

Same call surface as the reference (``pack_cuda.py:1040``, ``:1186``): inputs
are C-contiguous float32 ``(E, n, 3)`` CUDA arrays (torch tensors, or any
DLPack array such as a cupy array), outputs are caller-allocated and
overwritten, the functions return ``None``.  Arguments are validated on
every call (the reference does it only at ``debugging_mode >= 2``) and raise
``ValueError`` like the reference's checks.

Periodic images (``crystal_axes`` (E, 4) = [ax, ay, bx, by],
``only_self_interactions``, ``N_periodic``; ``pack_cuda.py:332-364``) run in
a kernel of their own (``pk_overlap_crystal``) with the reference's rules:
images of a tree itself count half and carry no gradient, ``only_self``
keeps only those at full weight, and with ``only_self_interactions`` but no
axes the result is zero.  Distinct ``xyt1``/``xyt2`` arrays raise
``NotImplementedError`` (every caller passes one array).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

MAX_PIECES = 4
MAX_VERTS_PER_PIECE = 4
MAX_INTERSECTION_VERTS = 8


def _same_array(a: torch.Tensor, b: torch.Tensor) -> bool:
    return a.data_ptr() == b.data_ptr() and a.shape == b.shape and a.dtype == b.dtype


def overlap_multi_ensemble(xyt1, xyt2, use_separation, out_cost=None, out_grads=None, crystal_axes=None,
                           only_self_interactions=False, N_periodic=2, stream=None):
    """Total overlap area (``use_separation=False``) or sum of squared SAT
    penetration depths (``True``) over all tree pairs of each ensemble, and
    optionally its gradient w.r.t. every pose.  Reference:
    ``pack_cuda.py:1040-1183`` (kernel ``multi_overlap_list_total`` :482)."""
    if not isinstance(use_separation, bool) and type(use_separation).__name__ != "bool_":
        raise ValueError("use_separation must be a boolean")
    x1 = _lib.as_tensor(xyt1, "xyt1")
    x2 = _lib.as_tensor(xyt2, "xyt2")
    if x1.ndim != 3 or x1.shape[2] != 3:
        raise ValueError(f"xyt1 must be shape (n_ensembles, n_trees, 3), got {tuple(x1.shape)}")
    _lib.check_f32(x1, "xyt1")
    _lib.check_f32(x2, "xyt2")
    if not _same_array(x1, x2):
        raise NotImplementedError("xyt1 and xyt2 must be the same array (every caller passes one array)")
    E, n = int(x1.shape[0]), int(x1.shape[1])
    if out_cost is None:
        raise ValueError("out_cost must be provided")
    c = _lib.as_tensor(out_cost, "out_cost")
    _lib.check_f32(c, "out_cost", (E,))
    g = None
    if out_grads is not None:
        g = _lib.as_tensor(out_grads, "out_grads")
        _lib.check_f32(g, "out_grads", (E, n, 3))
    ax = None
    if crystal_axes is not None:
        ax = _lib.as_tensor(crystal_axes, "crystal_axes")
        _lib.check_f32(ax, "crystal_axes", (E, 4))
        if not isinstance(N_periodic, (int,)) or N_periodic < 0:
            raise ValueError("N_periodic must be a non-negative int")
    if E == 0:
        return
    if ax is None and only_self_interactions:
        # no periodic images: no self interactions (pack_cuda.py:1061-1062)
        c.zero_()
        if g is not None:
            g.zero_()
        return
    _lib.ensure_init(x1.device)
    with torch.cuda.device(x1.device):
        sh = ctypes.c_void_p(_lib.stream_handle(stream, x1.device))
        if ax is None:
            rc = _lib.load().pk_overlap(_lib.ptr(x1), E, n, int(bool(use_separation)), _lib.ptr(c), _lib.ptr(g), sh)
        else:
            rc = _lib.load().pk_overlap_crystal(_lib.ptr(x1), E, n, int(bool(use_separation)), _lib.ptr(ax),
                                                int(bool(only_self_interactions)), int(N_periodic), _lib.ptr(c),
                                                _lib.ptr(g), sh)
    _lib.check(rc, "overlap_multi_ensemble")


def boundary_distance_multi_ensemble(xyt, h, out_cost=None, out_grads=None, out_grad_h=None, stream=None):
    """Sum over trees of the largest squared distance of a tree vertex
    outside the square ``[-h0/2, h0/2]^2 + (h1, h2)``, with gradients w.r.t.
    poses and h.  Reference: ``pack_cuda.py:1186-1295`` (kernel :706)."""
    x = _lib.as_tensor(xyt, "xyt")
    hh = _lib.as_tensor(h, "h")
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError(f"xyt must be shape (n_ensembles, n_trees, 3), got {tuple(x.shape)}")
    _lib.check_f32(x, "xyt")
    E, n = int(x.shape[0]), int(x.shape[1])
    if hh.ndim != 2 or hh.shape[1] != 3:
        raise ValueError(f"h must be shape (n_ensembles, 3), got {tuple(hh.shape)}")
    _lib.check_f32(hh, "h", (E, 3))
    if out_cost is None:
        raise ValueError("out_cost must be provided")
    c = _lib.as_tensor(out_cost, "out_cost")
    _lib.check_f32(c, "out_cost", (E,))
    g = gh = None
    if out_grads is not None:
        g = _lib.as_tensor(out_grads, "out_grads")
        _lib.check_f32(g, "out_grads", (E, n, 3))
    if out_grad_h is not None:
        gh = _lib.as_tensor(out_grad_h, "out_grad_h")
        _lib.check_f32(gh, "out_grad_h", (E, 3))
    if E == 0:
        return
    _lib.ensure_init(x.device)
    with torch.cuda.device(x.device):
        rc = _lib.load().pk_boundary(_lib.ptr(x), _lib.ptr(hh), E, n, _lib.ptr(c), _lib.ptr(g), _lib.ptr(gh),
                                     ctypes.c_void_p(_lib.stream_handle(stream, x.device)))
    _lib.check(rc, "boundary_distance_multi_ensemble")
