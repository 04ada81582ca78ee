"""pk_relax_noalloc: the relaxation entry point for callers that cannot
allocate device memory while they run (code under stream capture, hosts that
own every device byte through their own allocator, latency-bound loops where
cudaMalloc would synchronise the device).  Its L-BFGS history lives in an
array built into the library; its results must equal pk_relax's, which
takes a caller-allocated history buffer.  Called straight through the C ABI.
Collected last on purpose (test_zz_*): it also runs after every other test."""
import ctypes

import pytest
import torch

from packing_b200 import _lib
from packing_b200.cost import CostSpec
from packing_b200.relax import RelaxParams, workspace_floats
from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu


def _run_both(L, xyt, h, spec, prm, dev):
    E, n = int(xyt.shape[0]), int(xyt.shape[1])
    cs, ps = spec.to_c(), prm.to_c()
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    outs = []
    for noalloc in (False, True):
        xo = torch.full_like(xyt, float("nan"))
        ho = torch.full_like(h, float("nan"))
        lo = torch.full((E,), float("nan"), device=dev)
        it = torch.full((E,), -7, dtype=torch.int32, device=dev)
        if noalloc:
            rc = L.pk_relax_noalloc(_lib.ptr(xyt), _lib.ptr(h), E, n, ctypes.byref(cs), ctypes.byref(ps),
                                    _lib.ptr(xo), _lib.ptr(ho), _lib.ptr(lo), _lib.ptr(it), st)
        else:
            work = torch.empty(workspace_floats([n] * E, prm.history_size), device=dev)
            rc = L.pk_relax(_lib.ptr(xyt), _lib.ptr(h), None, None, E, n, ctypes.byref(cs), ctypes.byref(ps),
                            _lib.ptr(xo), _lib.ptr(ho), _lib.ptr(lo), _lib.ptr(it), _lib.ptr(work), st)
        assert rc == 0, L.pk_last_error()
        torch.cuda.synchronize(dev)
        outs.append((xo, ho, lo, it))
    return outs


def test_noalloc_matches_allocating_entry_point(cuda):
    L = _lib.load()
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)
    # two calls in a row with different batches: the built-in array keeps the
    # first call's history, which must not leak into the second call
    for seed, (E, n, hist, iters) in [(1, (48, 60, 8, 40)), (2, (32, 100, 5, 25))]:
        xyt = torch.from_numpy(poses(E, n, seed=seed)).to(cuda)
        h = torch.from_numpy(square_h(E, n)).to(cuda)
        prm = RelaxParams(n_iterations=iters, history_size=hist, max_step=0.01)
        (xa, ha, la, ia), (xb, hb, lb, ib) = _run_both(L, xyt, h, spec, prm, cuda)
        assert torch.all(ia == iters) and torch.equal(ia, ib)
        # the same kernel and the same arithmetic on both paths, with only the
        # history's address differing: the results agree bit for bit
        assert torch.equal(xb, xa)
        assert torch.equal(lb, la)
        assert torch.equal(hb, ha)


def test_noalloc_rejects_batches_beyond_its_array(cuda):
    L = _lib.load()
    spec = CostSpec(pair="area").to_c()
    prm = RelaxParams(n_iterations=5, history_size=10).to_c()
    E, n = 2048, 200          # 2 * 10 * 2048 * 603 floats > 4 Mi floats
    x = torch.zeros((1, n, 3), device=cuda)
    rc = L.pk_relax_noalloc(_lib.ptr(x), None, E, n, ctypes.byref(spec), ctypes.byref(prm), _lib.ptr(x), None,
                            _lib.ptr(x), None, None)
    assert rc == -4
    assert b"history floats" in L.pk_last_error()
