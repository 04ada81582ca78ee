"""Launch shapes of the fused relaxation: threads per packing and the
persistent grid change the speed, never the result; the launch can be
captured into a CUDA graph and replayed on new inputs; the autotuner picks
a feasible shape and caches it."""
import numpy as np
import pytest
import torch

from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu


def _spec():
    from packing_b200.cost import CostSpec
    return CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)


def _run(xyt, h, prm, offsets=None, order=None, n_max=None):
    from packing_b200.relax import relax_into, workspace_floats
    sizes = [xyt.shape[1]] * xyt.shape[0] if offsets is None else list(np.diff(offsets.cpu().numpy()))
    E = len(sizes)
    xo, ho = torch.empty_like(xyt), torch.empty_like(h)
    loss = torch.empty(E, device=xyt.device)
    it = torch.empty(E, dtype=torch.int32, device=xyt.device)
    work = torch.empty(workspace_floats(sizes, prm.history_size), device=xyt.device)
    relax_into(xyt, h, xo, ho, loss, work, _spec(), prm, offsets=offsets, order=order, n_max=n_max, iters_out=it)
    torch.cuda.synchronize()
    return xo.cpu().numpy(), loss.cpu().numpy(), it.cpu().numpy()


def test_threads_and_persistent_do_not_change_results(cuda):
    from packing_b200.relax import RelaxParams
    from packing_b200.tune import feasible_threads
    E, n = 37, 60
    xyt = torch.from_numpy(poses(E, n, seed=3)).to(cuda)
    h = torch.from_numpy(square_h(E, n)).to(cuda)
    ref = _run(xyt, h, RelaxParams(n_iterations=40, history_size=6, max_step=0.01))
    for t in [32] + feasible_threads(n):
        for p in (False, True):
            out = _run(xyt, h, RelaxParams(n_iterations=40, history_size=6, max_step=0.01, threads=t, persistent=p))
            for a, b in zip(ref, out):
                assert np.array_equal(a, b), (t, p)


def test_ragged_persistent_matches_one_cta_per_packing(cuda):
    from packing_b200.relax import RelaxParams
    rng = np.random.default_rng(5)
    sizes = [int(s) for s in rng.integers(5, 90, size=300)]
    flat = np.concatenate([poses(1, s, seed=100 + k)[0] for k, s in enumerate(sizes)]).astype(np.float32)
    off = np.zeros(len(sizes) + 1, np.int32)
    off[1:] = np.cumsum(sizes)
    h = np.concatenate([square_h(1, s) for s in sizes]).astype(np.float32)
    xt = torch.from_numpy(flat).to(cuda)
    ht = torch.from_numpy(h).to(cuda)
    offt = torch.from_numpy(off).to(cuda)
    order = torch.tensor(sorted(range(len(sizes)), key=lambda e: -sizes[e]), dtype=torch.int32, device=cuda)
    a = _run(xt, ht, RelaxParams(n_iterations=30, history_size=4), offsets=offt, order=order, n_max=max(sizes))
    b = _run(xt, ht, RelaxParams(n_iterations=30, history_size=4, persistent=True, threads=96), offsets=offt,
             order=order, n_max=max(sizes))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_graph_capture_and_replay(cuda):
    """The persistent launch captured once and replayed on new poses equals
    eager launches on the same poses."""
    from packing_b200.relax import RelaxParams, relax_into, workspace_floats
    E, n = 64, 50
    prm = RelaxParams(n_iterations=25, history_size=5, max_step=0.01, persistent=True)
    x_static = torch.from_numpy(poses(E, n, seed=21)).to(cuda)
    h_static = torch.from_numpy(square_h(E, n)).to(cuda)
    xo, ho = torch.empty_like(x_static), torch.empty_like(h_static)
    loss = torch.empty(E, device=cuda)
    it = torch.empty(E, dtype=torch.int32, device=cuda)
    work = torch.empty(workspace_floats([n] * E, prm.history_size), device=cuda)
    side = torch.cuda.Stream(cuda)
    side.wait_stream(torch.cuda.current_stream(cuda))
    with torch.cuda.stream(side):   # warm-up off the capture: attributes and occupancy are set here
        relax_into(x_static, h_static, xo, ho, loss, work, _spec(), prm, iters_out=it)
    torch.cuda.current_stream(cuda).wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        relax_into(x_static, h_static, xo, ho, loss, work, _spec(), prm, iters_out=it)
    for seed in (22, 23):
        new = torch.from_numpy(poses(E, n, seed=seed)).to(cuda)
        x_static.copy_(new)
        g.replay()
        torch.cuda.synchronize()
        got = (xo.cpu().numpy(), loss.cpu().numpy(), it.cpu().numpy())
        ref = _run(new, h_static, RelaxParams(n_iterations=25, history_size=5, max_step=0.01))
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    del g


def test_tuner_picks_feasible_shape_and_caches(cuda, tmp_path):
    from packing_b200.tune import RelaxTuner, feasible_threads
    tn = RelaxTuner(cuda, cache_path=str(tmp_path / "tune.json"), iterations=3, reps=1)
    t, p = tn.best(40, _spec(), 5)
    assert t in feasible_threads(48) and isinstance(p, bool)
    tn2 = RelaxTuner(cuda, cache_path=str(tmp_path / "tune.json"))

    def boom(*a, **k):
        raise AssertionError("cached shape was re-measured")
    tn2.measure = boom
    assert tn2.best(45, _spec(), 5) == (t, p)   # same bucket, read from the cache file
    prm = tn2.tuned(__import__("packing_b200.relax", fromlist=["RelaxParams"]).RelaxParams(history_size=5), 45,
                    _spec())
    assert prm.threads == t and prm.persistent == p


def _ragged(cuda, sizes, seed=0):
    flat = np.concatenate([poses(1, s, seed=seed + k)[0] for k, s in enumerate(sizes)]).astype(np.float32)
    off = np.zeros(len(sizes) + 1, np.int32)
    off[1:] = np.cumsum(sizes)
    h = np.concatenate([square_h(1, s) for s in sizes]).astype(np.float32)
    order_h = sorted(range(len(sizes)), key=lambda e: -sizes[e])
    return (torch.from_numpy(flat).to(cuda), torch.from_numpy(h).to(cuda), torch.from_numpy(off).to(cuda),
            torch.tensor(order_h, dtype=torch.int32, device=cuda), [sizes[e] for e in order_h])


def test_size_classes_match_one_launch(cuda):
    """One launch per size class, side by side on forked streams, gives the
    bits of one launch for the whole ragged batch."""
    from packing_b200.relax import RelaxParams, relax_into, size_classes, workspace_floats
    rng = np.random.default_rng(8)
    sizes = [int(s) for s in np.round(np.exp(rng.uniform(np.log(3), np.log(300), size=400)))]
    xt, ht, offt, order, in_order = _ragged(cuda, sizes, seed=500)
    prm = RelaxParams(n_iterations=30, history_size=5, max_step=0.01)
    ref = _run(xt, ht, prm, offsets=offt, order=order, n_max=max(sizes))
    classes = size_classes(in_order)
    assert len(classes) >= 5
    E = len(sizes)
    xo, ho = torch.empty_like(xt), torch.empty_like(ht)
    loss = torch.empty(E, device=cuda)
    it = torch.empty(E, dtype=torch.int32, device=cuda)
    work = torch.empty(workspace_floats(sizes, prm.history_size), device=cuda)
    relax_into(xt, ht, xo, ho, loss, work, _spec(), prm, offsets=offt, order=order, n_max=max(sizes),
               iters_out=it, classes=classes)
    torch.cuda.synchronize()
    for a, b in zip(ref, (xo.cpu().numpy(), loss.cpu().numpy(), it.cpu().numpy())):
        assert np.array_equal(a, b)


def test_size_classes_in_a_cuda_graph(cuda):
    """The class launches and their stream fork / join captured in one CUDA
    graph and replayed on new poses equal eager single launches."""
    from packing_b200.relax import RelaxParams, relax_into, size_classes, workspace_floats
    sizes = [7, 150, 33, 90, 12, 64, 200, 3, 48, 17] * 6
    xt, ht, offt, order, in_order = _ragged(cuda, sizes, seed=900)
    prm = RelaxParams(n_iterations=20, history_size=4, max_step=0.01)
    classes = size_classes(in_order)
    E = len(sizes)
    xo, ho = torch.empty_like(xt), torch.empty_like(ht)
    loss = torch.empty(E, device=cuda)
    work = torch.empty(workspace_floats(sizes, prm.history_size), device=cuda)
    side = torch.cuda.Stream(cuda)
    side.wait_stream(torch.cuda.current_stream(cuda))
    with torch.cuda.stream(side):   # warm-up off the capture
        relax_into(xt, ht, xo, ho, loss, work, _spec(), prm, offsets=offt, order=order, n_max=max(sizes),
                   classes=classes)
    torch.cuda.current_stream(cuda).wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        relax_into(xt, ht, xo, ho, loss, work, _spec(), prm, offsets=offt, order=order, n_max=max(sizes),
                   classes=classes)
    for seed in (901, 902):
        new, _, _, _, _ = _ragged(cuda, sizes, seed=seed)
        xt.copy_(new)
        g.replay()
        torch.cuda.synchronize()
        ref = _run(new, ht, prm, offsets=offt, order=order, n_max=max(sizes))
        assert np.array_equal(xo.cpu().numpy(), ref[0])
        assert np.array_equal(loss.cpu().numpy(), ref[1])
    del g


def test_partial_order_rejects_bad_counts(cuda):
    import ctypes
    from packing_b200 import _lib
    from packing_b200.relax import RelaxParams
    L = _lib.load()
    cs, ps = _spec().to_c(), RelaxParams().to_c()
    x = torch.zeros(30, device=cuda)
    o = torch.zeros(4, dtype=torch.int32, device=cuda)
    args = (_lib.ptr(x), _lib.ptr(x), None)
    rc = L.pk_relax_ordered(*args, _lib.ptr(o), 5, 4, 10, ctypes.byref(cs), ctypes.byref(ps), _lib.ptr(x), None,
                            _lib.ptr(x), None, _lib.ptr(x), None)
    assert rc != 0   # count above E
    rc = L.pk_relax_ordered(*args, None, 2, 4, 10, ctypes.byref(cs), ctypes.byref(ps), _lib.ptr(x), None,
                            _lib.ptr(x), None, _lib.ptr(x), None)
    assert rc != 0   # no order


def test_relax_into_refuses_short_or_wrong_buffers(cuda):
    """The kernel writes through raw pointers, so relax_into checks every
    caller buffer before launching: a history workspace one float short, an
    output of the wrong size or dtype, or a buffer on the host is a
    ValueError, and nothing is launched."""
    from packing_b200.relax import RelaxParams, relax_into, workspace_floats
    E, n = 4, 30
    xyt = torch.from_numpy(poses(E, n, seed=3)).to(cuda)
    h = torch.from_numpy(square_h(E, n)).to(cuda)
    prm = RelaxParams(n_iterations=5, history_size=4, max_step=0.01)
    need = workspace_floats([n] * E, 4)
    ok = dict(xyt_out=torch.empty_like(xyt), h_out=torch.empty_like(h), loss_out=torch.empty(E, device=cuda),
              work=torch.empty(need, device=cuda))
    relax_into(xyt, h, ok["xyt_out"], ok["h_out"], ok["loss_out"], ok["work"], _spec(), prm)
    bad = [dict(ok, work=torch.empty(need - 1, device=cuda)),
           dict(ok, loss_out=torch.empty(E - 1, device=cuda)),
           dict(ok, xyt_out=torch.empty((E, n + 1, 3), device=cuda)),
           dict(ok, xyt_out=torch.empty_like(xyt, dtype=torch.float64)),
           dict(ok, h_out=torch.empty((E - 1, 3), device=cuda)),
           dict(ok, work=torch.empty(need))]
    for b in bad:
        with pytest.raises(ValueError):
            relax_into(xyt, h, b["xyt_out"], b["h_out"], b["loss_out"], b["work"], _spec(), prm)
    with pytest.raises(ValueError):
        relax_into(xyt, h, ok["xyt_out"], ok["h_out"], ok["loss_out"], ok["work"], _spec(), prm,
                   iters_out=torch.empty(E, dtype=torch.int64, device=cuda))
