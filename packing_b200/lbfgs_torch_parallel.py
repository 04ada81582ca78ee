"""Drop-in for ``core/lbfgs_torch_parallel.py``: batched L-BFGS whose vector
algebra runs in three CUDA kernels per iteration instead of ~100-150 torch
launches and ~25 host synchronisations.

``lbfgs(func, x0, ...)`` keeps the reference's signature, defaults and
semantics (``lbfgs_torch_parallel.py:411-729``): ``func(x, is_main)`` returns
``(cost (M,), grad (M, N))``; ``x0`` (M, N) float32 or float64 on a CUDA
device is updated in place and returned.  Per iteration: direction kernel
(two-loop recursion, first-step scaling, ``max_step`` clamp, ``g.d`` stop) ->
one host read of "any system active" -> step kernel -> ``func`` -> history /
convergence kernel.  Inactive systems keep stepping while any system of the
batch is active, as in the reference.

``line_search_fn='strong_wolfe'`` (``:70-407``) is not provided: production
runs without line search (``pack_dynamics.py:39``); it raises
``NotImplementedError``.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch
from torch import Tensor

from . import _lib

__all__ = ["lbfgs"]


def lbfgs(func, x0: Tensor, lr: float = 1.0, max_iter: int = 20, max_eval: Optional[int] = None,
          tolerance_grad: float = 1e-7, tolerance_change: float = 1e-9, tolerance_rel_change: float = 0.,
          stop_on_cost_increase: bool = False, history_size: int = 100, line_search_fn: Optional[str] = None,
          max_step: Optional[float] = 0.5):
    if line_search_fn is not None:
        raise NotImplementedError("line_search_fn='strong_wolfe' is not provided by the CUDA drop-in")
    if max_eval is None:
        max_eval = max_iter * 5 // 4
    if not isinstance(x0, Tensor) or not x0.is_cuda:
        raise ValueError("x0 must be a CUDA tensor")
    if x0.dtype not in (torch.float32, torch.float64):
        raise ValueError("x0 must be float32 or float64")
    if x0.ndim != 2:
        raise ValueError("x0 must be (M, N)")
    M, N = x0.shape
    dev, dt = x0.device, x0.dtype
    m = int(history_size)
    x = x0.detach().clone().contiguous()

    def call(xx):
        loss, g = func(xx, True)
        loss = _lib.as_tensor(loss, "cost").to(dt).reshape(M).contiguous()
        g = _lib.as_tensor(g, "grad").to(dt).reshape(M, N).contiguous()
        return loss, g

    loss, g = call(x)
    loss = loss.clone()
    g = g.clone()
    if M == 0:
        return x0
    z = lambda *s: torch.zeros(*s, dtype=dt, device=dev)   # noqa: E731
    zi = lambda *s: torch.zeros(*s, dtype=torch.int32, device=dev)   # noqa: E731
    d, pg = z(M, N), z(M, N)
    ploss, loss0 = z(M), z(M)
    S, Y, ro = z(M, m, N), z(M, m, N), z(M, m)
    H, t = z(M), z(M)
    hlen, hstart, evals, active = zi(M), zi(M), zi(M), zi(M)
    flag = zi(1)
    host_flag = torch.zeros(1, dtype=torch.int32, pin_memory=True)
    L = _lib.load()
    nbytes = 4 if dt == torch.float32 else 8
    arrays_t = [x, g, loss, d, pg, ploss, loss0, S, Y, ro, H, t, hlen, hstart, evals, active, flag]

    def ptrs():
        return (ctypes.c_void_p * 17)(*[a.data_ptr() for a in arrays_t])

    arr = ptrs()

    def phase(p, n_iter, p0=0.0, p1=0.0, p2=0.0, i1=0, i2=0):
        with torch.cuda.device(dev):
            rc = L.pk_lbfgs_phase(p, nbytes, arr, M, N, m, n_iter, float(p0), float(p1), float(p2), 0.0, int(i1),
                                  int(i2), ctypes.c_void_p(_lib.stream_handle(None, dev)))
        _lib.check(rc, "lbfgs")

    def any_active() -> bool:
        host_flag.copy_(flag, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return bool(host_flag.item())

    flag.zero_()
    phase(0, 0, tolerance_grad)
    if not any_active():
        x0.copy_(x)
        return x0
    has_ms = max_step is not None
    n_iter = 0
    while n_iter < max_iter:
        n_iter += 1
        flag.zero_()
        phase(1, n_iter, lr, max_step if has_ms else 0.0, tolerance_change, i1=int(has_ms))
        if not any_active():
            break
        phase(2, n_iter)
        if n_iter != max_iter:
            nl, ng = call(x)
            loss.copy_(nl)
            g.copy_(ng)
        phase(3, n_iter, tolerance_grad, tolerance_change, tolerance_rel_change, i1=int(stop_on_cost_increase),
              i2=max_eval)
    x0.copy_(x)
    return x0
