"""Fused compound cost: one launch computes what ``CostCompound`` assembles
from separate kernels and cupy sums (``core/pack_cost.py:245-277``).

``compound_cost(xyt, h, ...)`` returns ``(cost (E,), grad (E, n, 3),
grad_h (E, 3))`` for ``w_area * h0^2 (zero with a fixed side, as AreaCost) + w_boundary * boundary + w_pair *
pairs``, the form of ``OptimizerBFGS``'s default cost
(``core/pack_dynamics.py:45-51``: AreaCost 1e-2, BoundaryDistanceCost 1,
CollisionCostOverlappingArea 1).  Ragged batches go through ``offsets``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib


@dataclass
class CostSpec:
    """Weights and pair term of a compound cost.  pair: 'area' | 'sep' |
    'lut' | 'none'.  ``lut`` is a ``pack_cuda_lut.LookupTable`` for 'lut'."""
    pair: str = "area"
    w_pair: float = 1.0
    w_boundary: float = 1.0
    w_area: float = 1e-2
    fixed_h: bool = True
    lut: object = None
    symmetry: int = 1   # 1: every tree given; 2 / 4: genotype of a 180 / 90 degree symmetric packing

    def to_c(self) -> _lib.PkCostSpec:
        s = _lib.PkCostSpec()
        modes = {"none": _lib.PK_PAIR_NONE, "area": _lib.PK_PAIR_AREA, "sep": _lib.PK_PAIR_SEP,
                 "lut": _lib.PK_PAIR_LUT}
        if self.pair not in modes:
            raise ValueError(f"pair must be one of {sorted(modes)}")
        s.pair_mode = modes[self.pair]
        s.w_pair = float(self.w_pair)
        s.w_boundary = float(self.w_boundary)
        s.w_area = float(self.w_area)
        s.fixed_h = int(bool(self.fixed_h))
        if self.symmetry not in (1, 2, 4):
            raise ValueError("symmetry must be 1, 2 or 4")
        s.symmetry = int(self.symmetry)
        if self.pair == "lut":
            if self.lut is None:
                raise ValueError("pair='lut' needs a LookupTable")
            s.lut = self.lut.c_struct()
        return s


def compound_cost(xyt, h, spec: CostSpec = CostSpec(), offsets=None, n_max=None, out_cost=None,
                  out_grad=None, out_grad_h=None, evaluate_gradient=True, stream=None, order=None, classes=None):
    """Fused compound cost and gradient.  Uniform batch: ``xyt`` (E, n, 3).
    Ragged batch: ``xyt`` (sum n, 3) with int32 ``offsets`` (E+1,) on the
    device and ``n_max`` >= every instance's tree count; with a largest-first
    ``order`` and its ``classes`` (``classes.ragged_plan``), one launch per
    size class side by side, bit-identical to one launch."""
    x = _lib.as_tensor(xyt, "xyt")
    _lib.check_f32(x, "xyt")
    if offsets is None:
        if x.ndim != 3 or x.shape[2] != 3:
            raise ValueError(f"xyt must be shape (E, n, 3), got {tuple(x.shape)}")
        E, n = int(x.shape[0]), int(x.shape[1])
        nm = n
        off = None
    else:
        off = _lib.as_tensor(offsets, "offsets")
        if off.dtype != torch.int32 or off.ndim != 1 or not off.is_cuda:
            raise ValueError("offsets must be a CUDA int32 vector (E+1,)")
        if x.ndim != 2 or x.shape[1] != 3:
            raise ValueError("ragged xyt must be shape (sum n, 3)")
        E = int(off.shape[0]) - 1
        if n_max is None:
            n_max = int((off[1:] - off[:-1]).max().item()) if E > 0 else 0
        nm = int(n_max)
    hh = None
    if h is not None:
        hh = _lib.as_tensor(h, "h")
        _lib.check_f32(hh, "h", (E, 3))
    dev = x.device
    cost = out_cost if out_cost is not None else torch.empty(E, device=dev, dtype=torch.float32)
    grad = grad_h = None
    if evaluate_gradient:
        grad = out_grad if out_grad is not None else torch.empty_like(x)
        if hh is not None:
            grad_h = out_grad_h if out_grad_h is not None else torch.empty_like(hh)
    if E == 0:
        return cost, grad, grad_h
    _lib.ensure_init(dev)
    cs = spec.to_c()
    if classes is not None:
        launch_cost_classes(x, off, order, E, nm, hh, cs, cost, grad, grad_h, classes, stream, "compound_cost")
        return cost, grad, grad_h
    with torch.cuda.device(dev):
        rc = _lib.load().pk_cost(_lib.ptr(x), _lib.ptr(off), E, nm, _lib.ptr(hh), ctypes.byref(cs),
                                 _lib.ptr(cost), _lib.ptr(grad), _lib.ptr(grad_h),
                                 ctypes.c_void_p(_lib.stream_handle(stream, dev)))
    _lib.check(rc, "compound_cost")
    return cost, grad, grad_h


def launch_cost_classes(x, off, order, E, n_max, h, cs, cost, grad, grad_h, classes, stream, what):
    """One pk_cost_ordered launch per size class, side by side on forked streams."""
    from .classes import launch_classes
    if off is None or order is None:
        raise ValueError(f"{what}: classes need a ragged batch with a largest-first order")
    if sum(c.count for c in classes) != E or any(c.n_max > n_max for c in classes):
        raise ValueError(f"{what}: classes must cover the order once, each within n_max")
    L = _lib.load()

    def launch(c, st):
        rc = L.pk_cost_ordered(_lib.ptr(x), _lib.ptr(off), ctypes.c_void_p(order.data_ptr() + 4 * c.start), c.count,
                               E, c.n_max, _lib.ptr(h), ctypes.byref(cs), int(c.threads), _lib.ptr(cost),
                               _lib.ptr(grad), _lib.ptr(grad_h), ctypes.c_void_p(st))
        _lib.check(rc, what)

    with torch.cuda.device(x.device):
        launch_classes(x.device, stream, classes, launch)
