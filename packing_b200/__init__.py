"""packing_b200 -- B200 (sm_100a) implementation of the jcottaar/packing hot
path: batched tree-pair cost and gradient, batched L-BFGS, batched Hungarian.

Drop-in modules keep the reference's module names and call surfaces:

* ``packing_b200.pack_cuda``            (core/pack_cuda.py)
* ``packing_b200.pack_cuda_lut``        (core/pack_cuda_lut.py)
* ``packing_b200.lap_batch``            (core/lap_batch.py)
* ``packing_b200.lbfgs_torch_parallel`` (core/lbfgs_torch_parallel.py)

B200-native additions: ``cost.compound_cost`` (fused CostCompound),
``relax.relax`` / ``relax.relax_ragged`` (one-launch batched relaxation),
``validate`` (FP64 legality), ``serve`` (continuous-batching relaxation
service).  All compute runs in ``libpackb200.so`` (``csrc/``), reached
through the C ABI declared in ``include/packb200.h``.
"""
from . import _lib  # noqa: F401

__version__ = "0.1.0"


def load():
    """Load the native library (building it first if stale)."""
    return _lib.load()
