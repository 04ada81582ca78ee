"""Batched legalisation of relaxed packings on the GPU: the B200 form of
``core/pack_io.py:28-112`` (``legalize``) with ``snap``
(``core/kaggle_support.py:824-879``) and the FP64 legality check that stands
in for the Kaggle metric's (``core/pack_metric.py:127-147``).

Per packing, as the reference does for one solution:

1. snap: trees re-centred on their bounding box, ``h = (min(side, h0), 0, 0)``
   and the side made free (``use_fixed_h = False``);
2. up to ``n_iter`` rounds of the fused relaxation of
   ``AreaCost(w) + BoundaryDistanceCost + CollisionCostSeparation`` (the GA's
   fitness cost with its collision term replaced, ``pack_io.py:61-64``,
   ``pack_ga3.py:1475-1477``), halving ``w`` from 1e-2 and shrinking
   ``max_step`` by sqrt(1/2) from 1e-4 each round; 20000 iterations in the
   first round and ``round(200 move_factor)`` after, history 10, no line
   search;
3. stop once boundary + separation cost is below ``target``;
4. FP64 validation; packings that fail are legalised once more with
   ``tolerance_rel_change = 0`` (``:105-112``).

The packings are batched: every round relaxes, in one launch, the packings
still above the target, and each packing's rounds depend on it alone, so its
result is the one it would get legalised alone.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .cost import CostSpec, compound_cost
from .relax import RelaxParams, relax
from .validate import validate


def snap(xyt, h=None, stream=None):
    """(xyt_snapped, h_snapped) of float32 packings (E, n, 3) and optional
    h (E, 3): re-centred trees and h = (min(side, h0), 0, 0)."""
    x = _lib.as_tensor(xyt, "xyt").contiguous()
    _lib.check_f32(x, "xyt")
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError("xyt must be (E, n, 3)")
    E, n = int(x.shape[0]), int(x.shape[1])
    hh = None
    if h is not None:
        hh = _lib.as_tensor(h, "h").contiguous()
        _lib.check_f32(hh, "h", (E, 3))
    xo = torch.empty_like(x)
    ho = torch.empty((E, 3), dtype=torch.float32, device=x.device)
    if E == 0:
        return xo, ho
    _lib.ensure_init(x.device)
    with torch.cuda.device(x.device):
        rc = _lib.load().pk_snap(_lib.ptr(x), _lib.ptr(hh), E, n, _lib.ptr(xo), _lib.ptr(ho),
                                 ctypes.c_void_p(_lib.stream_handle(stream, x.device)))
    _lib.check(rc, "snap")
    return xo, ho


@dataclass
class LegalizeResult:
    xyt: torch.Tensor          # (E, n, 3) legalised poses
    h: torch.Tensor            # (E, 3) square parameters after the rounds
    legal: torch.Tensor        # (E,) bool: no FP64 overlap
    side: torch.Tensor         # (E,) float64 side of the bounding square (legality tree)
    rounds: torch.Tensor       # (E,) int32 relaxation rounds used
    overlap_cost: torch.Tensor  # (E,) boundary + separation cost at the end


def _overlap_cost(xyt, h):
    spec = CostSpec(pair="sep", w_pair=1.0, w_boundary=1.0, w_area=0.0, fixed_h=False)
    c, _, _ = compound_cost(xyt, h, spec, evaluate_gradient=False)
    return c


def legalize(xyt, h=None, move_factor=10.0, tolerance_rel_change=1e-7, stop_on_cost_increase=False, n_iter=20,
             target=1e-10, validate_result=True, first_iterations=20000, verbose=False, _retry=True) -> LegalizeResult:
    """Legalise a batch of packings (E, n, 3) float32; see the module text."""
    x = _lib.as_tensor(xyt, "xyt").contiguous()
    _lib.check_f32(x, "xyt")
    E, n = int(x.shape[0]), int(x.shape[1])
    dev = x.device
    xs, hs = snap(x, h)
    rounds = torch.zeros(E, dtype=torch.int32, device=dev)
    todo = torch.arange(E, device=dev)
    w_area, max_step, iters = 1e-2, 1e-4, int(first_iterations)
    for _ in range(int(n_iter)):
        if todo.numel() == 0:
            break
        w_area *= 0.5
        max_step *= float(np.sqrt(0.5))
        spec = CostSpec(pair="sep", w_pair=1.0, w_boundary=1.0, w_area=w_area, fixed_h=False)
        prm = RelaxParams(n_iterations=iters, history_size=10, max_step=max_step,
                          tolerance_rel_change=tolerance_rel_change, stop_on_cost_increase=stop_on_cost_increase)
        xo, ho, _, _ = relax(xs.index_select(0, todo), hs.index_select(0, todo), spec, prm)
        xs.index_copy_(0, todo, xo)
        hs.index_copy_(0, todo, ho)
        rounds.index_add_(0, todo, torch.ones_like(todo, dtype=torch.int32))
        iters = int(np.round(200 * move_factor))
        oc = _overlap_cost(xo, ho)
        if verbose:
            print(f"legalize round {int(rounds.max())}: {todo.numel()} packings relaxed, overlap cost "
                  f"max {float(oc.max()):.3e}, {int((oc < target).sum())} below {target:g}")
        todo = todo[oc >= target]
    oc = _overlap_cost(xs, hs)
    if validate_result:
        ov, side = validate(xs)
        legal = ov == 0
    else:
        side = validate(xs)[1]
        legal = oc < target
    if _retry and tolerance_rel_change != 0.0 and not bool(legal.all()):
        bad = torch.nonzero(~legal).squeeze(1)
        r = legalize(xs.index_select(0, bad), hs.index_select(0, bad), move_factor, 0.0, stop_on_cost_increase,
                     n_iter, target, validate_result, first_iterations, verbose, _retry=False)
        xs.index_copy_(0, bad, r.xyt)
        hs.index_copy_(0, bad, r.h)
        legal = legal.clone()
        legal[bad] = r.legal
        side = side.clone()
        side[bad] = r.side
        rounds.index_add_(0, bad, r.rounds)
        oc = oc.clone()
        oc[bad] = r.overlap_cost
    return LegalizeResult(xs, hs, legal, side, rounds, oc)
