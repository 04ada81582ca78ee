"""Size classes of ragged batches.

One launch for a ragged batch gives every CTA the threads and shared memory
of its largest packing; small packings then spend their time at barriers.
A largest-first launch order splits into contiguous classes of tree counts,
and each class is launched with CTAs sized for its own trees, the classes
side by side on streams forked from the caller's stream and joined back to
it.  Every reduction's order depends on the packing alone, so the results
are those of one launch, bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib


@dataclass(frozen=True)
class SizeClass:
    """A contiguous part of a largest-first launch order: ``count`` instances
    from position ``start``, none with more than ``n_max`` trees, launched
    with CTAs of ``threads`` threads (0: the library default for ``n_max``)."""
    start: int
    count: int
    n_max: int
    threads: int


# (largest tree count, threads per CTA) of the size classes: a class's CTA
# has about as many threads as its largest packing has trees, from 32 to 256.
# Chosen by timing class tables on a ragged batch of 8192 packings with n
# log-uniform in [5, 200] (C4) on a B200: the relaxations (area and LUT cost)
# and the one-shot LUT cost kernel.  Splitting the old 140 -> 160 class at 120
# (128 threads) and giving 121-160 trees 192 threads made the LUT cost kernel
# 4 % and the area relaxation 1 % faster, the LUT relaxation unchanged.
CLASS_TABLE = ((20, 32), (40, 64), (80, 96), (120, 128), (160, 192), (256, 256), (512, 256), (1024, 256))
CLASS_EDGES = tuple(e for e, _ in CLASS_TABLE)


def size_classes(sizes_in_order) -> list[SizeClass]:
    """Size classes of a ragged batch, given its tree counts in the launch
    order (largest first).  A packing of n trees goes to the class of the
    smallest edge >= n in ``CLASS_TABLE``, whose CTAs have that entry's
    threads."""
    sz = [int(v) for v in sizes_in_order]
    if any(sz[k] < sz[k + 1] for k in range(len(sz) - 1)):
        raise ValueError("sizes must be in a largest-first order")
    out, k = [], 0
    while k < len(sz):
        edge = next((e for e in CLASS_EDGES if sz[k] <= e), None)
        if edge is None:
            raise ValueError(f"{sz[k]} trees exceeds {CLASS_EDGES[-1]}")
        lo = max([e for e in CLASS_EDGES if e < edge], default=0)
        j = k
        while j < len(sz) and sz[j] > lo:
            j += 1
        out.append(SizeClass(start=k, count=j - k, n_max=sz[k], threads=dict(CLASS_TABLE)[edge]))
        k = j
    return out


def ragged_plan(sizes, device=None):
    """(order, classes) for a ragged batch with these tree counts: the
    largest-first launch order as a device int32 tensor and its size
    classes."""
    order_h = sorted(range(len(sizes)), key=lambda e: -int(sizes[e]))
    order = torch.tensor(order_h, dtype=torch.int32, device=device or "cuda")
    return order, size_classes([int(sizes[e]) for e in order_h])


_side_streams: dict[int, list] = {}


def side_streams(dev, k):
    """k side streams of a device (created once, reused)."""
    d = _lib._dev_index(dev)
    lst = _side_streams.setdefault(d, [])
    while len(lst) < k:
        lst.append(torch.cuda.Stream(device=torch.device("cuda", d)))
    return lst[:k]


def base_stream(stream, dev):
    """The torch stream of a stream argument (None: the current stream)."""
    if stream is None:
        return torch.cuda.current_stream(dev)
    if isinstance(stream, torch.cuda.Stream):
        return stream
    return torch.cuda.ExternalStream(_lib.stream_handle(stream, dev), device=dev)


def launch_classes(dev, stream, classes, launch):
    """Call launch(cls, stream_handle) for every class, each on its own side
    stream forked from ``stream`` (None: the current stream) and joined back
    to it."""
    base = base_stream(stream, dev)
    side = side_streams(dev, len(classes))
    fork = torch.cuda.Event()
    fork.record(base)
    for c, st in zip(classes, side):
        st.wait_event(fork)
        launch(c, st.cuda_stream)
        join = torch.cuda.Event()
        join.record(st)
        base.wait_event(join)
