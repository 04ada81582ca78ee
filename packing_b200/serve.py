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
  side by side on forked streams;
* the host never waits for the step the GPU is running: up to ``depth``
  steps are queued on the stream, each followed by an asynchronous copy of
  the job table into its own pinned snapshot.  While step k runs, the host
  reads step k-1's snapshot, queues the gather and copy-back of the jobs it
  finished, and admits waiting requests into the slots and pool ranges they
  freed -- all stream-ordered behind the work that still reads them.  A job
  finished on the device is skipped by later steps until the host retires it;
* a job's result does not depend on its neighbours or its chunking (order-
  fixed reductions, pause at iteration boundaries), so it equals the result
  of relaxing it alone.

``RelaxServer.submit`` queues a request; ``step`` runs one engine step to
completion; ``drain`` and ``run_trace`` keep the pipeline full, and
``run_trace`` replays an arrival trace in real time and reports p50/p99
latency (arrival to the result on the host) and throughput.
"""
from __future__ import annotations

import collections
import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .cost import CostSpec
from .classes import CLASS_EDGES, CLASS_TABLE, SizeClass, launch_classes
from .relax import RelaxParams

_JOB_BYTES = ctypes.sizeof(_lib.PkJob)
# PkJob as a numpy record (the C struct's field order and alignment), so a
# batch of admitted jobs is filled without a Python loop over ctypes objects
_JOB_DTYPE = np.dtype([("n", "i4"), ("max_iter", "i4"), ("x_off", "i8"), ("h_off", "i8"), ("status", "i4"),
                       ("it", "i4"), ("evals", "i4"), ("hlen", "i4"), ("hstart", "i4"), ("H", "f4"),
                       ("loss", "f4"), ("loss0", "f4")], align=True)
assert _JOB_DTYPE.itemsize == _JOB_BYTES


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
        self.release_many([(off, n)])

    def release_many(self, ranges):
        for off, n in ranges:
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


def _classes_of(sizes: np.ndarray) -> list[SizeClass]:
    """classes.size_classes for a largest-first numpy array of tree counts,
    with vector operations."""
    edges = np.array(CLASS_EDGES)
    if len(sizes) and sizes[0] > edges[-1]:
        raise ValueError(f"{int(sizes[0])} trees exceeds {int(edges[-1])}")
    cls = np.searchsorted(edges, sizes, side="left")          # class of each job
    bounds = np.flatnonzero(np.diff(cls)) + 1
    starts = np.concatenate([[0], bounds])
    ends = np.concatenate([bounds, [len(sizes)]])
    threads = dict(CLASS_TABLE)
    return [SizeClass(int(a), int(b - a), int(sizes[a]), threads[int(edges[cls[a]])]) for a, b in zip(starts, ends)]


class RelaxServer:
    def __init__(self, spec: CostSpec = CostSpec(), history: int = 10, max_step: float = 0.01,
                 chunk_iters: int = 16, pool_floats: int = 1 << 27, max_jobs: int = 8192, device=None,
                 classes: bool = True, depth: int = 2):
        self.dev = torch.device(device or "cuda")
        _lib.ensure_init(self.dev)
        self.spec_c = spec.to_c()
        self.params = RelaxParams(n_iterations=1, history_size=history, max_step=max_step)
        self.m = history
        self.chunk = int(chunk_iters)
        self.pool = torch.empty(pool_floats, dtype=torch.float32, device=self.dev)
        self.alloc = _Pool(pool_floats)
        self.max_jobs = max_jobs
        self.depth = max(1, int(depth))
        # the device job table; host-side entries are only ever written for
        # newly admitted slots (running jobs' entries live on the device)
        self.table_d = torch.zeros((max_jobs, _JOB_BYTES), dtype=torch.uint8, device=self.dev)
        # one pinned snapshot of the table per step that can be in flight
        self.snaps = [torch.empty((max_jobs, _JOB_BYTES), dtype=torch.uint8).pin_memory()
                      for _ in range(self.depth + 1)]
        self._snap_next = 0
        self.free_slots = list(range(max_jobs - 1, -1, -1))
        self.pending: collections.deque[Request] = collections.deque()
        # per-slot state of the resident jobs, as arrays so that a step over
        # thousands of jobs costs the host a few vector operations
        self.slot_req: list[Request | None] = [None] * max_jobs
        self.slot_gen = np.zeros(max_jobs, dtype=np.int64)    # admissions into the slot so far
        self.slot_n = np.zeros(max_jobs, dtype=np.int64)
        self.slot_off = np.zeros(max_jobs, dtype=np.int64)
        self.slot_need = np.zeros(max_jobs, dtype=np.int64)
        self.res = np.zeros(max_jobs, dtype=bool)
        self.inflight: collections.deque = collections.deque()    # (event, snapshot, slots, gens, list)
        self.retiring: collections.deque = collections.deque()    # (event, host buffer, [(req, n, pos)])
        self.done: list[Request] = []
        self.launches = 0
        self._next_id = 0
        self.stream = torch.cuda.current_stream(self.dev)
        self.classes = bool(classes)

    @property
    def resident(self) -> dict[int, Request]:
        """slot -> request of every job holding pool memory."""
        return {int(k): self.slot_req[k] for k in np.flatnonzero(self.res)}

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

    def _h2d(self, arr: np.ndarray) -> torch.Tensor:
        """Stream-ordered copy of a host array through pinned memory (the
        caching host allocator keeps the buffer until the copy has run)."""
        t = torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
        return t.to(self.dev, non_blocking=True)

    def _admit(self):
        """Admit what fits: one copy + scatter for every admitted job's x =
        [xyt, h], one copy + scatter for their table entries."""
        slots, offs, ns, its, vals = [], [], [], [], []
        while self.pending and self.free_slots:
            req = self.pending[0]
            need = self.footprint(req.xyt.shape[0])
            off = self.alloc.alloc(need)
            if off is None:
                break   # memory-based admission: wait until running jobs free their footprint
            self.pending.popleft()
            slot = self.free_slots.pop()
            slots.append(slot)
            offs.append(off)
            ns.append(req.xyt.shape[0])
            its.append(req.iters)
            vals.append(req.xyt.reshape(-1))
            vals.append(req.h)
            self.slot_req[slot] = req
            self.slot_need[slot] = need
        if slots:
            sl = np.array(slots, dtype=np.int64)
            offs_a, ns_a = np.array(offs, dtype=np.int64), np.array(ns, dtype=np.int64)
            self.slot_gen[sl] += 1
            self.slot_n[sl], self.slot_off[sl] = ns_a, offs_a
            self.res[sl] = True
            N = 3 * ns_a + 3
            rec = np.zeros(len(slots), dtype=_JOB_DTYPE)
            rec["n"], rec["max_iter"], rec["x_off"] = ns_a, its, offs_a
            rec["h_off"] = offs_a + 2 * N + self.m
            rec["status"], rec["evals"], rec["H"] = _lib.PK_JOB_NEW, 1, 1.0
            # pool positions of every job's x = [xyt, h]: off .. off + N
            ii = np.repeat(offs_a - np.concatenate([[0], np.cumsum(N)[:-1]]), N) + np.arange(int(N.sum()))
            with torch.cuda.stream(self.stream):
                self.pool.index_copy_(0, self._h2d(ii), self._h2d(np.concatenate(vals).astype(np.float32)))
                self.table_d.index_copy_(0, self._h2d(sl), self._h2d(rec.view(np.uint8).reshape(len(slots),
                                                                                                  _JOB_BYTES)))
        return slots

    def _launch(self):
        """Queue one engine step over every resident job, then the table
        snapshot and an event."""
        slots = np.flatnonzero(self.res)
        slots = slots[np.argsort(-self.slot_n[slots], kind="stable")]
        sizes = self.slot_n[slots]
        lst = self._h2d(slots.astype(np.int32))
        classes = _classes_of(sizes) if self.classes else [SizeClass(0, len(slots), int(sizes[0]), 0)]
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
            snap = self.snaps[self._snap_next]
            self._snap_next = (self._snap_next + 1) % len(self.snaps)
            with torch.cuda.stream(self.stream):
                snap.copy_(self.table_d, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.stream)
        self.launches += 1
        # the jobs this step ran, with their admission counts: a slot freed and
        # given to a new job after the step was queued still shows the old
        # job's entry in this snapshot
        self.inflight.append((ev, snap, slots, self.slot_gen[slots].copy(), lst))

    def _collect(self, block: bool) -> int:
        """Read the oldest completed step's snapshot: queue the gather and
        copy-back of the jobs it finished and free their slots and pool ranges
        (later work on the stream runs after the gather).  Returns the number
        of steps collected."""
        k = 0
        while self.inflight:
            ev, snap, slots, gens, _ = self.inflight[0]
            if not block and not ev.query():
                break
            ev.synchronize()
            self.inflight.popleft()
            k += 1
            block = False
            tab = snap.numpy().view(_JOB_DTYPE).reshape(-1)
            fin = slots[self.res[slots] & (self.slot_gen[slots] == gens) & (tab["status"][slots] == _lib.PK_JOB_DONE)]
            if len(fin) == 0:
                continue
            lens = 3 * self.slot_n[fin] + 3
            starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
            pos = int(lens.sum())
            ii = np.repeat(self.slot_off[fin] - starts, lens) + np.arange(pos)
            items = []
            for s, p0, loss, it in zip(fin.tolist(), starts.tolist(), tab["loss"][fin].tolist(),
                                       tab["it"][fin].tolist()):
                req = self.slot_req[s]
                req.loss, req.iterations = float(loss), int(it)
                items.append((req, req.xyt.shape[0], p0))
                self.slot_req[s] = None
            self.res[fin] = False
            self.alloc.release_many(zip(self.slot_off[fin].tolist(), self.slot_need[fin].tolist()))
            self.free_slots.extend(fin.tolist())
            with torch.cuda.stream(self.stream):
                xs = self.pool.index_select(0, self._h2d(ii))
                host = torch.empty(pos, dtype=torch.float32).pin_memory()
                host.copy_(xs, non_blocking=True)
                ev2 = torch.cuda.Event()
                ev2.record(self.stream)
            self.retiring.append((ev2, host, items))
        return k

    def _finish(self, block: bool) -> list[Request]:
        """Hand over the results whose copy-back has completed."""
        out = []
        while self.retiring:
            ev, host, items = self.retiring[0]
            if not block and not ev.query():
                break
            ev.synchronize()
            self.retiring.popleft()
            block = False
            now = time.perf_counter()
            x = host.numpy()
            for req, n, pos in items:
                req.result = x[pos:pos + 3 * n].reshape(n, 3).copy()
                req.h_out = x[pos + 3 * n:pos + 3 * n + 3].copy()
                req.t_done = now
                out.append(req)
        self.done.extend(out)
        return out

    def timed_step(self):
        """step() with the engine launches timed on the device (CUDA events
        around the size-class launches): (completed requests, seconds)."""
        self._collect(block=True)
        self._admit()
        if not self.res.any():
            return self._finish(block=True), 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        self._launch()
        e1.record(self.stream)
        self._collect(block=True)
        out = self._finish(block=True)
        return out, e0.elapsed_time(e1) / 1e3

    def _busy(self) -> bool:
        return bool(self.pending or self.res.any() or self.inflight or self.retiring)

    def step(self) -> list[Request]:
        """Admit what fits, advance every resident job by one chunk, retire
        the finished ones, and wait for all of it.  Returns the requests
        completed by this step."""
        self._collect(block=True)
        self._admit()
        if self.res.any():
            self._launch()
        self._collect(block=True)
        return self._finish(block=True)

    def _pump(self):
        """One turn of the pipelined loop: collect what the GPU has finished,
        keep up to ``depth`` steps queued, wait only when nothing else can be
        done."""
        self._collect(block=False)
        self._finish(block=False)
        if (self.pending or self.res.any()) and len(self.inflight) < self.depth:
            self._admit()
            if self.res.any():
                self._launch()
                return
        if self.inflight:
            self._collect(block=True)
        elif self.retiring:
            self._finish(block=True)

    def drain(self):
        while self._busy():
            self._pump()
        return self.done

    # ------------------------------------------------------------------
    def run_trace(self, requests, arrival_times):
        """Replay arrivals (seconds from start, non-decreasing) in real time.
        requests: list of (xyt, h, iters).  Returns latency statistics."""
        t0 = time.perf_counter()
        order = list(zip(arrival_times, requests))
        k = 0
        reqs = []
        while k < len(order) or self._busy():
            now = time.perf_counter() - t0
            while k < len(order) and order[k][0] <= now:
                ta, (xyt, h, iters) = order[k]
                reqs.append(self.submit(xyt, h, iters, t_arrival=t0 + ta))
                k += 1
            if not self._busy() and k < len(order):
                time.sleep(max(0.0, min(order[k][0] - now, 0.001)))
                continue
            self._pump()
        wall = time.perf_counter() - t0
        lat = np.array([r.t_done - r.t_arrival for r in reqs])
        return {"requests": len(reqs), "wall_s": wall, "relaxations_per_s": len(reqs) / wall,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3), "launches": self.launches}, reqs
