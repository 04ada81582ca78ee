"""Fused batched relaxation: the B200 form of ``OptimizerBFGS.run_simulation``
(``core/pack_dynamics.py:54-149``) over ``lbfgs`` (``lbfgs_torch_parallel.py:411``).

One CUDA launch relaxes a whole batch: each CTA owns one packing, keeps its
parameters ``x = [xyt (3n), h (3)]``, gradient and search direction in
shared memory, evaluates the compound cost with the cost kernel's device code
and runs all L-BFGS iterations without returning to the host.  Ragged
batches (different tree counts) go largest first, either in one launch or as
one launch per size class with CTAs sized for that class's trees, the
classes side by side on forked streams.  ``relax_into`` does no host
synchronisation and no allocation, so it can be captured in a CUDA graph.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from .classes import CLASS_EDGES, CLASS_TABLE, SizeClass, launch_classes, size_classes  # noqa: F401
from .cost import CostSpec


PkRelaxParams = _lib.PkRelaxParams


@dataclass
class RelaxParams:
    """OptimizerBFGS defaults (pack_dynamics.py:33-39) with lbfgs's own
    defaults for what pack_dynamics passes explicitly (tolerances 0)."""
    n_iterations: int = 100
    history_size: int = 3
    max_step: float | None = 0.01
    lr: float = 1.0
    tolerance_grad: float = 0.0
    tolerance_change: float = 0.0
    tolerance_rel_change: float = 0.0
    stop_on_cost_increase: bool = False
    max_eval: int | None = None
    final_eval: bool = True
    counters: object = None      # optional CUDA int64 tensor (6,), accumulated work counts
    threads: int = 0             # threads per packing (0: library default; see tune.py)
    persistent: bool = False     # one CTA per resident slot instead of one per packing

    def to_c(self) -> PkRelaxParams:
        p = PkRelaxParams()
        p.max_iter = int(self.n_iterations)
        p.history = int(self.history_size)
        p.lr = float(self.lr)
        p.has_max_step = int(self.max_step is not None)
        p.max_step = float(self.max_step or 0.0)
        p.tol_grad = float(self.tolerance_grad)
        p.tol_change = float(self.tolerance_change)
        p.tol_rel_change = float(self.tolerance_rel_change)
        p.stop_on_cost_increase = int(bool(self.stop_on_cost_increase))
        p.max_eval = int(self.max_eval if self.max_eval is not None else self.n_iterations * 5 // 4)
        p.final_eval = int(bool(self.final_eval))
        p.counters = self.counters.data_ptr() if self.counters is not None else None
        p.threads = int(self.threads)
        p.persistent = int(bool(self.persistent))
        return p


def workspace_floats(sizes, history: int) -> int:
    """Floats of L-BFGS history scratch for a batch with these tree counts."""
    return 2 * int(history) * sum(3 * int(s) + 3 for s in sizes)


def _check_buffers(x, E, h, xyt_out, h_out, loss_out, iters_out, work, history):
    """The kernel writes through raw pointers: every caller buffer must be a
    contiguous CUDA array of the right type and at least the size the launch
    writes, or the launch is refused.  x is (E, n, 3) or ragged (sum n, 3), so
    x.numel() / 3 trees in either case."""
    trees = x.numel() // 3

    def need(t, name, dtype, numel, exact=False):
        if t is None:
            raise ValueError(f"{name} is required")
        t = _lib.as_tensor(t, name)
        if not t.is_cuda or t.device != x.device:
            raise ValueError(f"{name} must be on {x.device}")
        if t.dtype != dtype:
            raise ValueError(f"{name} must have dtype {dtype}, got {t.dtype}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be C-contiguous")
        if t.numel() < numel or (exact and t.numel() != numel):
            raise ValueError(f"{name} holds {t.numel()} elements; the launch writes {numel}")

    need(xyt_out, "xyt_out", torch.float32, x.numel(), exact=True)
    need(loss_out, "loss_out", torch.float32, E)
    need(work, "work", torch.float32, 2 * int(history) * (3 * trees + 3 * E))
    if h is not None:
        need(h, "h", torch.float32, 3 * E)
    if h_out is not None:
        need(h_out, "h_out", torch.float32, 3 * E)
    if iters_out is not None:
        need(iters_out, "iters_out", torch.int32, E)


def relax_into(xyt, h, xyt_out, h_out, loss_out, work, spec: CostSpec, params: RelaxParams, offsets=None,
               order=None, n_max=None, iters_out=None, stream=None, classes=None):
    """Launch the fused relaxation on caller-provided buffers (no host sync,
    no allocation).  Uniform: xyt (E, n, 3).  Ragged: xyt (sum n, 3) with
    device int32 offsets (E+1,) and n_max.

    ``classes`` (ragged, with a largest-first ``order``): a list of
    ``SizeClass`` covering the order (``size_classes``).  Each class is one
    ``pk_relax_ordered`` launch with CTAs sized for its own trees, on its own
    stream forked from ``stream`` and joined back to it, so small packings
    do not hold CTAs sized for the largest.  Results are the same bit for
    bit as one launch."""
    x = _lib.as_tensor(xyt, "xyt")
    _lib.check_f32(x, "xyt")
    if offsets is None:
        if x.ndim != 3 or x.shape[2] != 3:
            raise ValueError(f"xyt must be shape (E, n, 3), got {tuple(x.shape)}")
        E, nm = int(x.shape[0]), int(x.shape[1])
    else:
        if x.ndim != 2 or x.shape[1] != 3:
            raise ValueError(f"ragged xyt must be shape (sum n, 3), got {tuple(x.shape)}")
        if n_max is None:
            raise ValueError("a ragged batch needs n_max")
        E = int(offsets.shape[0]) - 1
        nm = int(n_max)
    _check_buffers(x, E, h, xyt_out, h_out, loss_out, iters_out, work, params.history_size)
    dev = x.device
    cs = spec.to_c()
    L = _lib.load()
    if classes is None:
        ps = params.to_c()
        with torch.cuda.device(dev):
            rc = L.pk_relax(_lib.ptr(x), _lib.ptr(h), _lib.ptr(offsets), _lib.ptr(order), E, nm,
                            ctypes.byref(cs), ctypes.byref(ps), _lib.ptr(xyt_out), _lib.ptr(h_out),
                            _lib.ptr(loss_out), _lib.ptr(iters_out), _lib.ptr(work),
                            ctypes.c_void_p(_lib.stream_handle(stream, dev)))
        _lib.check(rc, "pk_relax")
        return
    if order is None or offsets is None:
        raise ValueError("classes need a ragged batch with a largest-first order")
    if sum(c.count for c in classes) != E or any(c.n_max > nm for c in classes):
        raise ValueError("classes must cover the order once, each within n_max")

    def launch(c, st):
        ps = params.to_c()
        ps.threads = int(c.threads)
        rc = L.pk_relax_ordered(_lib.ptr(x), _lib.ptr(h), _lib.ptr(offsets),
                                ctypes.c_void_p(order.data_ptr() + 4 * c.start), c.count, E, c.n_max,
                                ctypes.byref(cs), ctypes.byref(ps), _lib.ptr(xyt_out), _lib.ptr(h_out),
                                _lib.ptr(loss_out), _lib.ptr(iters_out), _lib.ptr(work), ctypes.c_void_p(st))
        _lib.check(rc, "pk_relax_ordered")

    with torch.cuda.device(dev):
        launch_classes(dev, stream, classes, launch)


def relax(xyt, h, spec: CostSpec = CostSpec(), params: RelaxParams = RelaxParams(), stream=None):
    """Relax a uniform batch (E, n, 3) with square parameters h (E, 3).
    Returns (xyt_out, h_out, loss (E,), iterations (E,))."""
    x = _lib.as_tensor(xyt, "xyt").contiguous()
    _lib.check_f32(x, "xyt")
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError("xyt must be (E, n, 3)")
    E, n = int(x.shape[0]), int(x.shape[1])
    hh = _lib.as_tensor(h, "h").contiguous() if h is not None else None
    if hh is not None:
        _lib.check_f32(hh, "h", (E, 3))
    dev = x.device
    _lib.ensure_init(dev)
    xo = torch.empty_like(x)
    ho = torch.empty_like(hh) if hh is not None else None
    loss = torch.empty(E, dtype=torch.float32, device=dev)
    iters = torch.empty(E, dtype=torch.int32, device=dev)
    work = torch.empty(max(1, workspace_floats([n] * E, params.history_size)), dtype=torch.float32, device=dev)
    if E > 0:
        relax_into(x, hh, xo, ho, loss, work, spec, params, iters_out=iters, stream=stream)
    return xo, ho, loss, iters


def relax_ragged(xyt_list, h, spec: CostSpec = CostSpec(), params: RelaxParams = RelaxParams(), stream=None):
    """Relax packings of different tree counts together, largest first:
    one launch per size class (``size_classes``), side by side on forked
    streams; with ``params.threads`` set, one launch for all.  xyt_list: list
    of (n_e, 3) CUDA tensors; h (E, 3).  Returns (list of relaxed (n_e, 3),
    h_out, loss (E,), iterations (E,))."""
    sizes = [int(a.shape[0]) for a in xyt_list]
    E = len(sizes)
    if E == 0:
        return [], None, None, None
    dev = xyt_list[0].device
    _lib.ensure_init(dev)
    flat = torch.cat([a.reshape(-1, 3).to(torch.float32) for a in xyt_list]).contiguous()
    off_h = [0]
    for s in sizes:
        off_h.append(off_h[-1] + s)
    offsets = torch.tensor(off_h, dtype=torch.int32, device=dev)
    order_h = sorted(range(E), key=lambda e: -sizes[e])
    order = torch.tensor(order_h, dtype=torch.int32, device=dev)
    hh = _lib.as_tensor(h, "h").contiguous() if h is not None else None
    xo = torch.empty_like(flat)
    ho = torch.empty_like(hh) if hh is not None else None
    loss = torch.empty(E, dtype=torch.float32, device=dev)
    iters = torch.empty(E, dtype=torch.int32, device=dev)
    work = torch.empty(max(1, workspace_floats(sizes, params.history_size)), dtype=torch.float32, device=dev)
    classes = size_classes([sizes[e] for e in order_h]) if params.threads == 0 else None
    relax_into(flat, hh, xo, ho, loss, work, spec, params, offsets=offsets, order=order, n_max=max(sizes),
               iters_out=iters, stream=stream, classes=classes)
    outs = [xo[off_h[e]:off_h[e + 1]] for e in range(E)]
    return outs, ho, loss, iters
