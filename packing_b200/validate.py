"""Strict FP64 legality of packings and their bounding-square side.

``validate(xyt) -> (overlaps int32 (E,), side float64 (E,))``: the number of
tree pairs whose interiors intersect and the side of the smallest
axis-aligned square holding every tree, evaluated in double precision on the
legality tree -- the Kaggle metric's unexpanded tree (``core/pack_metric.py``
:27-79, :127-147) placed in the pose frame of the search tree
(``core/pack_io.py:150-158``).  Touching trees are legal, as in the metric.
A packing relaxed in FP32 is accepted only if this check finds no overlap.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib


def validate(xyt, stream=None):
    x = _lib.as_tensor(xyt, "xyt")
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError(f"xyt must be (E, n, 3), got {tuple(x.shape)}")
    if x.dtype not in (torch.float32, torch.float64) or not x.is_cuda:
        raise ValueError("xyt must be a float32 or float64 CUDA array")
    x = x.contiguous()
    E, n = int(x.shape[0]), int(x.shape[1])
    ov = torch.zeros(E, dtype=torch.int32, device=x.device)
    side = torch.zeros(E, dtype=torch.float64, device=x.device)
    if E == 0:
        return ov, side
    _lib.ensure_init(x.device)
    with torch.cuda.device(x.device):
        rc = _lib.load().pk_validate_fp64(_lib.ptr(x), x.element_size(), E, n, _lib.ptr(ov), _lib.ptr(side),
                                          ctypes.c_void_p(_lib.stream_handle(stream, x.device)))
    _lib.check(rc, "validate")
    return ov, side


def is_legal(xyt, stream=None) -> torch.Tensor:
    """Boolean (E,): no two trees of the packing overlap in FP64."""
    ov, _ = validate(xyt, stream)
    return ov == 0
