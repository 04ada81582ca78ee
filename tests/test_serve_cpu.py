"""Host-side pieces of the serving engine that need no GPU: the size-class
split of a step's jobs, the pool allocator, and the job record layout the
engine writes for the kernel."""
import ctypes

import numpy as np

from packing_b200 import _lib
from packing_b200.classes import size_classes
from packing_b200.serve import _JOB_DTYPE, _Pool, _classes_of


def test_vector_class_split_equals_size_classes():
    rng = np.random.default_rng(1)
    for _ in range(200):
        sz = np.sort(rng.integers(1, 600, size=int(rng.integers(1, 400))))[::-1]
        assert _classes_of(sz) == size_classes(sz.tolist())


def test_job_record_matches_the_c_struct():
    assert _JOB_DTYPE.itemsize == ctypes.sizeof(_lib.PkJob)
    rec = np.zeros(1, dtype=_JOB_DTYPE)
    vals = dict(n=5, max_iter=7, x_off=123456789012, h_off=9, status=2, it=3, evals=4, hlen=5, hstart=6, H=1.5,
                loss=2.5, loss0=3.5)
    for k, v in vals.items():
        rec[k] = v
    J = _lib.PkJob.from_buffer_copy(rec.tobytes())
    for k, v in vals.items():
        assert getattr(J, k) == v


def test_pool_first_fit_and_coalescing():
    p = _Pool(100)
    a, b, c = p.alloc(30), p.alloc(30), p.alloc(30)
    assert (a, b, c) == (0, 30, 60) and p.alloc(20) is None and p.used == 90
    p.release_many([(a, 30), (c, 30)])
    assert p.alloc(40) == 60            # the freed tail merged with the unused 10
    p.release(b, 30)
    assert p.free == [(0, 60)] and p.used == 40
