"""Autotuner for the fused relaxation's launch shape.

The relaxation kernel (``pk_relax``, one CTA per packing) can run with any
multiple of 32 threads per packing up to 256 and with either one CTA per
packing or a persistent grid of one CTA per resident slot.  Every reduction
in it has an order fixed by the packing alone, so the choice changes the
speed and never the result.  Which shape is fastest depends on the tree
count: shared memory per packing grows with n and sets how many CTAs fit on
an SM, and the pair work per packing grows with n^2.

``RelaxTuner.best(n_max, spec, history)`` times every feasible shape on a
synthetic batch of that tree count (seeded uniform poses at the solver's
density, the same square side rule as the GA's initial packings) and keeps
the fastest, per GPU model, tree-count bucket, pair term and history length,
in memory and in a JSON cache file.  ``tuned(params, n_max, spec)`` returns a
copy of a ``RelaxParams`` with the tuned shape filled in.
"""
from __future__ import annotations

import dataclasses
import json
import os
import threading

import numpy as np
import torch

from . import _lib
from .cost import CostSpec
from .relax import RelaxParams, relax_into, workspace_floats

CANDIDATE_THREADS = (64, 96, 128, 160, 192, 224, 256)
# tree-count buckets: a size is tuned at its bucket's upper edge
BUCKET_EDGES = (8, 16, 24, 32, 48, 64, 96, 128, 160, 200, 256, 320, 384, 512, 640, 768, 1024)
TREE_AREA = 0.2456875

_lock = threading.Lock()


def feasible_threads(n_max: int) -> list[int]:
    """Thread counts the kernel accepts for packings of up to n_max trees: its
    near-pair list (8 x threads entries) must hold one tree's n_max - 1 pairs."""
    return [t for t in CANDIDATE_THREADS if 8 * t >= n_max - 1]


def bucket(n_max: int) -> int:
    for e in BUCKET_EDGES:
        if n_max <= e:
            return e
    raise ValueError(f"n_max {n_max} exceeds {BUCKET_EDGES[-1]} trees")


def default_cache_path() -> str:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "packing_b200", "relax_tune.json")


def sample_batch(E: int, n: int, seed: int = 0):
    """Seeded packings of n trees: x, y uniform in a square of side
    1.3 sqrt(n * tree area), theta uniform; square side from the GA's rule
    sqrt((0.317 + 0.206 / sqrt(n)) n sqrt(1.1)) (pack_ga3.py:1136-1142)."""
    rng = np.random.default_rng(seed)
    s = 1.3 * np.sqrt(n * TREE_AREA)
    xy = rng.uniform(-s / 2, s / 2, size=(E, n, 2))
    th = rng.uniform(0.0, 2 * np.pi, size=(E, n, 1))
    h = np.zeros((E, 3), np.float32)
    h[:, 0] = np.sqrt((0.317 + 0.206 / np.sqrt(n)) * n * np.sqrt(1.1))
    return np.concatenate([xy, th], 2).astype(np.float32), h


class RelaxTuner:
    """Times launch shapes of the fused relaxation and remembers the best."""

    def __init__(self, device=None, cache_path: str | None = None, iterations: int = 6, reps: int = 2):
        self.device = torch.device("cuda", _lib._dev_index(device))
        self.cache_path = cache_path if cache_path is not None else default_cache_path()
        self.iterations = int(iterations)
        self.reps = int(reps)
        self.table: dict[str, dict] = {}
        self._load()

    def gpu_name(self) -> str:
        p = torch.cuda.get_device_properties(self.device)
        return f"{p.name}|sm{p.major}{p.minor}|{p.multi_processor_count}sm"

    def key(self, n_max: int, spec: CostSpec, history: int) -> str:
        sym = int(getattr(spec, "symmetry", 1) or 1)
        return f"{self.gpu_name()}|n{bucket(n_max)}|{spec.pair}|s{sym}|m{int(history)}"

    def _load(self):
        if self.cache_path and os.path.exists(self.cache_path):
            try:
                with open(self.cache_path) as f:
                    data = json.load(f)
                if isinstance(data, dict):
                    self.table.update({k: v for k, v in data.items() if isinstance(v, dict)})
            except (OSError, ValueError):
                pass   # an unreadable cache is retuned, not fatal

    def _save(self):
        if not self.cache_path:
            return
        try:
            os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
            tmp = self.cache_path + f".{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(self.table, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)
        except OSError:
            pass

    def candidates(self, n_max: int, symmetry: int = 1):
        return [(t, p) for t in feasible_threads(n_max * symmetry) for p in (False, True)]

    def measure(self, n_max: int, spec: CostSpec, history: int, E: int | None = None) -> dict:
        """Milliseconds per launch of every feasible shape on a sample batch
        of E packings of n_max trees (default: about eight waves of the GPU)."""
        _lib.ensure_init(self.device)
        dev = self.device
        if E is None:
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            E = int(min(4096, max(2 * sms, 8 * sms * max(1, 256 // max(n_max, 1)))))
        xyt_np, h_np = sample_batch(E, n_max, seed=1234)
        xyt = torch.from_numpy(xyt_np).to(dev)
        h = torch.from_numpy(h_np).to(dev)
        xo, ho = torch.empty_like(xyt), torch.empty_like(h)
        loss = torch.empty(E, device=dev)
        work = torch.empty(max(1, workspace_floats([n_max] * E, history)), device=dev)
        st = torch.cuda.current_stream(dev)
        out = {}
        for t, p in self.candidates(n_max, int(getattr(spec, "symmetry", 1) or 1)):
            prm = RelaxParams(n_iterations=self.iterations, history_size=history, max_step=0.01, final_eval=False,
                              threads=t, persistent=p)
            relax_into(xyt, h, xo, ho, loss, work, spec, prm)   # warm-up
            best = float("inf")
            for _ in range(self.reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                relax_into(xyt, h, xo, ho, loss, work, spec, prm)
                e1.record(st)
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
            out[(t, p)] = best
        return out

    def best(self, n_max: int, spec: CostSpec, history: int) -> tuple[int, bool]:
        """(threads, persistent) for packings of up to n_max trees: cached, or
        tuned now at the bucket's upper edge."""
        k = self.key(n_max, spec, history)
        with _lock:
            hit = self.table.get(k)
        if hit is None:
            nb = bucket(n_max)
            if nb * int(getattr(spec, "symmetry", 1) or 1) > 1024:   # the kernel's phenotype limit
                nb = n_max
            times = self.measure(nb, spec, history)
            (t, p), ms = min(times.items(), key=lambda kv: kv[1])
            hit = {"threads": int(t), "persistent": bool(p), "ms": ms, "n_tuned": nb,
                   "all_ms": {f"{tt}{'p' if pp else ''}": v for (tt, pp), v in times.items()}}
            with _lock:
                self.table[k] = hit
                self._save()
        return int(hit["threads"]), bool(hit["persistent"])

    def tuned(self, params: RelaxParams, n_max: int, spec: CostSpec) -> RelaxParams:
        t, p = self.best(n_max, spec, params.history_size)
        if 8 * t < n_max * int(getattr(spec, "symmetry", 1) or 1) - 1:   # feasible at the bucket's edge, so here
            t = 0
        return dataclasses.replace(params, threads=t, persistent=p)


_default: dict[int, RelaxTuner] = {}


def tuner(device=None) -> RelaxTuner:
    """The process-wide tuner of a device."""
    d = _lib._dev_index(device)
    with _lock:
        if d not in _default:
            _default[d] = RelaxTuner(d)
        return _default[d]


def tuned(params: RelaxParams, n_max: int, spec: CostSpec = CostSpec(), device=None) -> RelaxParams:
    return tuner(device).tuned(params, n_max, spec)
