"""Continuous-batching relaxation service on one GPU.

The reference relaxes offspring with ``pack_dynamics.run_simulation_list``
(``core/pack_dynamics.py:152-236``): it groups solutions by tree count and runs
one blocking L-BFGS per group, so work of different sizes never shares the
GPU and nothing new starts until the whole batch ends.  Here requests of any
tree count and iteration budget are served continuously:

* every admitted job keeps its poses, gradient and L-BFGS history resident in
  one device pool; admission is by memory footprint ((2 + 2m)(3n + 3) + m
  floats per job, first fit, FIFO);
* each engine step advances every resident job by ``chunk_iters``
  iterations with ``pk_relax_jobs``: the jobs go largest first, one launch
  per size class (``classes.size_classes``: CTAs sized for that class's trees)
  side by side on forked streams; then the step retires finished jobs and
  admits waiting ones -- requests that arrive while others run join at the
  next step and share launches with them;
* a job's result does not depend on its neighbours or its chunking (order-
  fixed reductions, pause at iteration boundaries), so it equals the result
  of relaxing it alone.

``RelaxServer.submit`` queues a request; ``step`` runs one engine step;
``run_trace`` replays an arrival trace in real time and reports p50/p99
latency and throughput.
"""
from __future__ import annotations

import collections
import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .cost import CostSpec
from .classes import SizeClass, launch_classes, size_classes
from .relax import RelaxParams


@dataclass
class Request:
    rid: int
    xyt: np.ndarray          # (n, 3) float32
    h: np.ndarray            # (3,) float32
    iters: int
    t_arrival: float = 0.0
    t_done: float = 0.0
    result: np.ndarray = None
    h_out: np.ndarray = None
    loss: float = float("nan")
    iterations: int = 0


class _Pool:
    """First-fit allocator over a float range with coalescing free list."""

    def __init__(self, size: int):
        self.size = size
        self.free = [(0, size)]
        self.used = 0

    def alloc(self, n: int):
        for k, (off, sz) in enumerate(self.free):
            if sz >= n:
                if sz == n:
                    self.free.pop(k)
                else:
                    self.free[k] = (off + n, sz - n)
                self.used += n
                return off
        return None

    def release(self, off: int, n: int):
        self.used -= n
        self.free.append((off, n))
        self.free.sort()
        merged = []
        for o, s in self.free:
            if merged and merged[-1][0] + merged[-1][1] == o:
                merged[-1] = (merged[-1][0], merged[-1][1] + s)
            else:
                merged.append((o, s))
        self.free = merged


class RelaxServer:
    def __init__(self, spec: CostSpec = CostSpec(), history: int = 10, max_step: float = 0.01,
                 chunk_iters: int = 16, pool_floats: int = 1 << 27, max_jobs: int = 8192, device=None,
                 classes: bool = True):
        self.dev = torch.device(device or "cuda")
        _lib.ensure_init(self.dev)
        self.spec_c = spec.to_c()
        self.params = RelaxParams(n_iterations=1, history_size=history, max_step=max_step)
        self.prm_c = self.params.to_c()
        self.m = history
        self.chunk = int(chunk_iters)
        self.pool = torch.empty(pool_floats, dtype=torch.float32, device=self.dev)
        self.alloc = _Pool(pool_floats)
        self.max_jobs = max_jobs
        self.table_h = (_lib.PkJob * max_jobs)()
        self.table_pin = torch.empty(ctypes.sizeof(self.table_h), dtype=torch.uint8).pin_memory()
        self.table_d = torch.empty(ctypes.sizeof(self.table_h), dtype=torch.uint8, device=self.dev)
        self.free_slots = list(range(max_jobs - 1, -1, -1))
        self.pending: collections.deque[Request] = collections.deque()
        self.resident: dict[int, tuple[Request, int, int]] = {}   # slot -> (req, off, floats)
        self.done: list[Request] = []
        self.launches = 0
        self._next_id = 0
        self.stream = torch.cuda.current_stream(self.dev)
        self.classes = bool(classes)

    # ------------------------------------------------------------------
    def footprint(self, n: int) -> int:
        N = 3 * n + 3
        return 2 * N + self.m + 2 * self.m * N

    def submit(self, xyt, h, iters: int, t_arrival: float | None = None) -> Request:
        xyt = np.ascontiguousarray(np.asarray(xyt, dtype=np.float32).reshape(-1, 3))
        n = xyt.shape[0]
        if n > _lib.PK_MAX_TREES:
            raise ValueError("more than 1024 trees")
        if self.footprint(n) > self.alloc.size:
            raise ValueError("request larger than the whole pool")
        req = Request(self._next_id, xyt, np.asarray(h, dtype=np.float32).reshape(3), int(iters),
                      time.perf_counter() if t_arrival is None else t_arrival)
        self._next_id += 1
        self.pending.append(req)
        return req

    def _admit(self):
        admitted = []
        idx, vals = [], []
        while self.pending and self.free_slots:
            req = self.pending[0]
            need = self.footprint(req.xyt.shape[0])
            off = self.alloc.alloc(need)
            if off is None:
                break   # memory-based admission: wait until running jobs free their footprint
            self.pending.popleft()
            slot = self.free_slots.pop()
            n = req.xyt.shape[0]
            N = 3 * n + 3
            J = self.table_h[slot]
            J.n, J.max_iter, J.x_off, J.h_off = n, req.iters, off, off + 2 * N + self.m
            J.status, J.it, J.evals, J.hlen, J.hstart = _lib.PK_JOB_NEW, 0, 1, 0, 0
            J.H, J.loss, J.loss0 = 1.0, 0.0, 0.0
            idx.append(np.arange(off, off + N, dtype=np.int64))
            vals.append(req.xyt.reshape(-1))
            vals.append(req.h)
            self.resident[slot] = (req, off, need)
            admitted.append(slot)
        if admitted:   # every admitted job's x = [xyt, h] in one copy and one scatter
            ii = torch.from_numpy(np.concatenate(idx)).to(self.dev)
            vv = torch.from_numpy(np.concatenate(vals).astype(np.float32)).to(self.dev)
            self.pool.index_copy_(0, ii, vv)
        return admitted

    def step(self) -> list[Request]:
        """Admit what fits, advance every resident job by one chunk, retire
        the finished ones.  Returns the requests completed by this step."""
        self._admit()
        if not self.resident:
            return []
        slots = sorted(self.resident, key=lambda s: -self.resident[s][0].xyt.shape[0])
        n_max = max(self.resident[s][0].xyt.shape[0] for s in slots)
        lst = torch.tensor(slots, dtype=torch.int32, device=self.dev)
        ctypes.memmove(self.table_pin.data_ptr(), ctypes.addressof(self.table_h), ctypes.sizeof(self.table_h))
        self.table_d.copy_(self.table_pin, non_blocking=True)
        sizes = [self.resident[s][0].xyt.shape[0] for s in slots]
        classes = size_classes(sizes) if self.classes else [SizeClass(0, len(slots), n_max, 0)]
        L = _lib.load()

        def launch(c, st):
            prm = self.params.to_c()
            prm.threads = int(c.threads)
            rc = L.pk_relax_jobs(ctypes.c_void_p(self.table_d.data_ptr()),
                                 ctypes.c_void_p(lst.data_ptr() + 4 * c.start), c.count, _lib.ptr(self.pool),
                                 c.n_max, ctypes.byref(self.spec_c), ctypes.byref(prm), self.chunk, ctypes.c_void_p(st))
            _lib.check(rc, "pk_relax_jobs")

        with torch.cuda.device(self.dev):
            launch_classes(self.dev, self.stream, classes, launch)
        self.launches += 1
        self.table_pin.copy_(self.table_d, non_blocking=True)
        self.stream.synchronize()
        ctypes.memmove(ctypes.addressof(self.table_h), self.table_pin.data_ptr(), ctypes.sizeof(self.table_h))
        finished = [s for s in slots if self.table_h[s].status == _lib.PK_JOB_DONE]
        out = []
        if finished:
            # every finished job's x = [xyt, h] in one gather and one copy
            spans = [(self.resident[s][1], 3 * self.resident[s][0].xyt.shape[0] + 3) for s in finished]
            ii = torch.from_numpy(np.concatenate([np.arange(o, o + k, dtype=np.int64) for o, k in spans]))
            allx = self.pool.index_select(0, ii.to(self.dev)).cpu().numpy()
            now = time.perf_counter()
            pos = 0
            for s in finished:
                req, off, need = self.resident.pop(s)
                n = req.xyt.shape[0]
                x = allx[pos:pos + 3 * n + 3]
                pos += 3 * n + 3
                req.result = x[:3 * n].reshape(n, 3).copy()
                req.h_out = x[3 * n:].copy()
                req.loss = float(self.table_h[s].loss)
                req.iterations = int(self.table_h[s].it)
                req.t_done = now
                self.alloc.release(off, need)
                self.free_slots.append(s)
                out.append(req)
            self.done.extend(out)
        return out

    def drain(self):
        while self.pending or self.resident:
            self.step()
        return self.done

    # ------------------------------------------------------------------
    def run_trace(self, requests, arrival_times):
        """Replay arrivals (seconds from start, non-decreasing) in real time.
        requests: list of (xyt, h, iters).  Returns latency statistics."""
        t0 = time.perf_counter()
        order = list(zip(arrival_times, requests))
        k = 0
        reqs = []
        while k < len(order) or self.pending or self.resident:
            now = time.perf_counter() - t0
            while k < len(order) and order[k][0] <= now:
                ta, (xyt, h, iters) = order[k]
                reqs.append(self.submit(xyt, h, iters, t_arrival=t0 + ta))
                k += 1
            if not self.pending and not self.resident and k < len(order):
                time.sleep(max(0.0, min(order[k][0] - now, 0.001)))
                continue
            self.step()
        wall = time.perf_counter() - t0
        lat = np.array([r.t_done - r.t_arrival for r in reqs])
        return {"requests": len(reqs), "wall_s": wall, "relaxations_per_s": len(reqs) / wall,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3), "launches": self.launches}, reqs
