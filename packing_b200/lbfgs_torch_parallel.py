"""Drop-in for ``core/lbfgs_torch_parallel.py``: batched L-BFGS whose vector
algebra runs in CUDA kernels instead of ~100-150 torch launches and ~25 host
synchronisations per iteration.

``lbfgs(func, x0, ...)`` keeps the reference's signature, defaults and
semantics (``lbfgs_torch_parallel.py:411-729``): ``func(x, is_main)`` returns
``(cost (M,), grad (M, N))``; ``x0`` (M, N) float32 or float64 on a CUDA
device is updated in place and returned.  Per iteration: direction kernel
(two-loop recursion, first-step scaling, ``max_step`` clamp, ``g.d`` stop) ->
one host read of "any system active" -> the step -> history / convergence
kernel.

* ``line_search_fn=None`` (production, ``pack_dynamics.py:39``): every system
  steps by ``t d`` while any system of the batch is active, then ``func`` is
  evaluated once (not on the last iteration), as in the reference.
* ``line_search_fn='strong_wolfe'``: the batched strong-Wolfe search
  (``_strong_wolfe_batched``, ``:70-407``) runs on the active systems as a
  device state machine (``pk_wolfe_phase``); between its phases ``func`` is
  called on exactly the rows the reference evaluates -- first all searched
  systems with ``is_main=True``, then the systems still searching with
  ``is_main=False`` -- so ``func`` sees the same calls.  Only the searched
  systems step, with the accepted step.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch
from torch import Tensor

from . import _lib

__all__ = ["lbfgs"]

# _strong_wolfe_batched's defaults, which the reference's main loop uses
# (lbfgs_torch_parallel.py:78-81, called at :613-617)
WOLFE_C1, WOLFE_C2, WOLFE_TOL_CHANGE, WOLFE_MAX_LS = 1e-4, 0.9, 1e-9, 25


class _WolfeSearch:
    """Device state of the batched strong-Wolfe search over M systems."""

    def __init__(self, L, M, N, dt, dev, x, d, g, loss, t, in_ls, evals):
        z = lambda *s: torch.zeros(*s, dtype=dt, device=dev)   # noqa: E731
        zi = lambda *s: torch.zeros(*s, dtype=torch.int32, device=dev)   # noqa: E731
        self.L, self.M, self.N, self.dev = L, M, N, dev
        self.nbytes = 4 if dt == torch.float32 else 8
        self.x, self.d, self.g, self.loss, self.t, self.in_ls, self.evals_main = x, d, g, loss, t, in_ls, evals
        self.gtd = z(M)
        self.x_new, self.g_new, self.f_new, self.gtd_new = z(M, N), z(M, N), z(M), z(M)
        self.g_prev, self.f_prev, self.gtd_prev, self.t_prev = z(M, N), z(M), z(M), z(M)
        self.bg, self.bt, self.bf, self.bgtd = z(M, 2, N), z(M, 2), z(M, 2), z(M, 2)
        self.d_norm, self.t_new = z(M), z(M)
        self.bsize, self.done, self.active, self.low, self.insuf, self.evals = (zi(M) for _ in range(6))
        self.flag = zi(1)
        self.host_flag = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        arrays = [x, d, g, loss, self.gtd, t, self.x_new, self.g_new, self.f_new, self.gtd_new, self.g_prev,
                  self.f_prev, self.gtd_prev, self.t_prev, self.bg, self.bt, self.bf, self.bgtd, self.d_norm,
                  self.t_new, self.bsize, self.done, self.active, self.low, self.insuf, self.evals, in_ls, self.flag]
        self._keep = arrays
        self.arr = (ctypes.c_void_p * len(arrays))(*[a.data_ptr() for a in arrays])

    def _phase(self, p, ls_iter=0, flag_arg=0):
        with torch.cuda.device(self.dev):
            rc = self.L.pk_wolfe_phase(p, self.nbytes, self.arr, self.M, self.N, int(ls_iter), WOLFE_C1, WOLFE_C2,
                                       WOLFE_TOL_CHANGE, int(flag_arg),
                                       ctypes.c_void_p(_lib.stream_handle(None, self.dev)))
        _lib.check(rc, "lbfgs strong_wolfe")

    def _any(self) -> bool:
        self.host_flag.copy_(self.flag, non_blocking=True)
        torch.cuda.current_stream(self.dev).synchronize()
        return bool(self.host_flag.item())

    def _evaluate(self, call, mask, is_main):
        rows = torch.nonzero((mask != 0) & (self.in_ls != 0)).squeeze(1)
        f_sub, g_sub = call(self.x_new.index_select(0, rows), is_main, int(rows.numel()))
        self.f_new.index_copy_(0, rows, f_sub)
        self.g_new.index_copy_(0, rows, g_sub)

    def run(self, call):
        self._phase(0)
        self._evaluate(call, self.in_ls, True)
        self._phase(1, flag_arg=1)
        ls_iter = 0
        while ls_iter < WOLFE_MAX_LS:           # bracketing (:146-233)
            self.flag.zero_()
            self._phase(2, ls_iter=ls_iter)
            if not self._any():
                break
            self._evaluate(call, self.active, False)
            self._phase(1)
            ls_iter += 1
        self._phase(3, flag_arg=int(ls_iter == WOLFE_MAX_LS))
        while ls_iter < WOLFE_MAX_LS:           # zoom (:260-389)
            self.flag.zero_()
            self._phase(4)
            if not self._any():
                break
            self._evaluate(call, self.active, False)
            self._phase(1)
            ls_iter += 1
            self._phase(5)
        self._phase(6)
        with torch.cuda.device(self.dev):
            rc = self.L.pk_wolfe_apply(self.nbytes, _lib.ptr(self.x), _lib.ptr(self.g), _lib.ptr(self.loss),
                                       _lib.ptr(self.evals_main), _lib.ptr(self.d), _lib.ptr(self.t),
                                       _lib.ptr(self.f_new), _lib.ptr(self.g_new), _lib.ptr(self.in_ls),
                                       _lib.ptr(self.evals), self.M, self.N,
                                       ctypes.c_void_p(_lib.stream_handle(None, self.dev)))
        _lib.check(rc, "lbfgs strong_wolfe")


def lbfgs(func, x0: Tensor, lr: float = 1.0, max_iter: int = 20, max_eval: Optional[int] = None,
          tolerance_grad: float = 1e-7, tolerance_change: float = 1e-9, tolerance_rel_change: float = 0.,
          stop_on_cost_increase: bool = False, history_size: int = 100, line_search_fn: Optional[str] = None,
          max_step: Optional[float] = 0.5):
    if line_search_fn not in (None, "strong_wolfe"):
        raise ValueError("line_search_fn must be None or 'strong_wolfe'")
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

    def call(xx, is_main=True, rows=M):
        loss, g = func(xx, is_main)
        loss = _lib.as_tensor(loss, "cost").to(dt).reshape(rows).contiguous()
        g = _lib.as_tensor(g, "grad").to(dt).reshape(rows, N).contiguous()
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

    search = _WolfeSearch(L, M, N, dt, dev, x, d, g, loss, t, active, evals) if line_search_fn else None
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
        if search is not None:
            search.run(call)
        else:
            phase(2, n_iter)
            if n_iter != max_iter:
                nl, ng = call(x)
                loss.copy_(nl)
                g.copy_(ng)
        phase(3, n_iter, tolerance_grad, tolerance_change, tolerance_rel_change, i1=int(stop_on_cost_increase),
              i2=max_eval)
    x0.copy_(x)
    return x0
