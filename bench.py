"""Benchmark: L-BFGS relaxations per second at n = 200.

Workload (one "step"): relax a population of E = 4096 packings of n = 200
trees (seeded uniform poses in a square of side 1.3 sqrt(n * tree area),
theta uniform in [0, 360) deg), history m = 10, 200 iterations, fixed square
side, cost = boundary distance + overlap area (+ 1e-2 h0^2, inactive with a
fixed side) -- OptimizerBFGS's default objective (pack_dynamics.py:45-51).
Synthetic data: the reference publishes no dataset.

ours (default): the fused one-launch relaxation (packing_b200.relax).  Also
  reported: e2e through the public API from pinned host buffers, the plain
  drop-in (reference-style lbfgs loop over the same cost kernel), the FP32
  roofline of the relaxation kernel, the CPU oracle baseline.
--impl reference: the reference's CPU implementation of the path, i.e. the
  FP64 C restatement of its cost kernels driven by the restatement of its
  lbfgs, on the host cores (the reference has no other CPU path that runs
  here: its own CPU cost needs shapely, which is absent).

Multi-GPU (torchrun): every rank relaxes its own E packings (weak scaling,
no data-path collective); value = all ranks' relaxations / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TREE_AREA = 0.2456875
METRIC = "L-BFGS relaxations/sec at n=200 (batched vs plain, same GPU); p50/p99 serve latency"


def workload(E, n, seed):
    rng = np.random.default_rng(seed)
    s = 1.3 * np.sqrt(n * TREE_AREA)
    xy = rng.uniform(-s / 2, s / 2, size=(E, n, 2))
    th = np.deg2rad(rng.uniform(0.0, 360.0, size=(E, n, 1)))
    xyt = np.concatenate([xy, th], 2).astype(np.float32)
    h = np.zeros((E, 3), np.float32)
    h[:, 0] = np.sqrt((0.317 + 0.206 / np.sqrt(n)) * n * np.sqrt(1.1))
    return xyt, h


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp32_peak_tflops(torch, L, dev):
    """Measured FP32 FMA throughput of this GPU (TFLOP/s), best of 5."""
    import ctypes
    props = torch.cuda.get_device_properties(dev)
    blocks, threads, iters = props.multi_processor_count * 8, 256, 20000
    out = torch.empty(blocks, device=dev)
    st = torch.cuda.current_stream(dev)
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rc = L.pk_fma_probe(ctypes.c_void_p(out.data_ptr()), blocks, threads, iters,
                            ctypes.c_void_p(st.cuda_stream))
        e1.record(st)
        torch.cuda.synchronize(dev)
        assert rc == 0
        ms = e0.elapsed_time(e1)
        best = max(best, blocks * threads * iters * 16 / (ms * 1e-3) / 1e12)
    return best


def gather_peak(torch, L, table, dev):
    """Measured trilinear lookups per second on uniformly random cells of
    ``table`` (nx, ny, nt) -- the LUT itself, so the same size and L2
    residency -- best of 5: the ceiling of the LUT cost kernel."""
    import ctypes
    props = torch.cuda.get_device_properties(dev)
    blocks, threads, iters = props.multi_processor_count * 8, 256, 32
    nx, ny, nt = (int(v) for v in table.shape)
    out = torch.empty(blocks, device=dev)
    st = torch.cuda.current_stream(dev)
    best = 0.0
    for k in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rc = L.pk_gather_probe(ctypes.c_void_p(table.data_ptr()), nx, ny, nt, ctypes.c_void_p(out.data_ptr()),
                               blocks, threads, iters, 7 + k, ctypes.c_void_p(st.cuda_stream))
        e1.record(st)
        torch.cuda.synchronize(dev)
        assert rc == 0
        if k:
            best = max(best, blocks * threads * iters * 2 / (e0.elapsed_time(e1) * 1e-3))
    return best


def cpu_baseline_relax(E, n, iters, history, seed=123):
    """The FP64 oracle relaxing a bounded sample of the same workload."""
    from oracle import oracle as O
    xyt, h = workload(E, n, seed)
    x0 = np.concatenate([xyt.reshape(E, -1), h], 1).astype(np.float64)

    def f(x):
        c, g, gh = O.compound_cost(x[:, :3 * n].reshape(E, n, 3), x[:, 3 * n:], w_area=1e-2, fixed_h=True)
        return c, np.concatenate([g.reshape(E, -1), gh], 1)

    t0 = time.perf_counter()
    O.lbfgs(f, x0, max_iter=iters, history_size=history, max_step=0.01, tolerance_grad=0, tolerance_change=0)
    dt = time.perf_counter() - t0
    return E / dt, O.num_threads(), dt


# Algorithmic FP32 work per counted unit, counted on the reference's own
# arithmetic by the oracle's op-counting mode (oracle.count_ops and
# oracle.lbfgs_ops; add / sub / mul / div / cmp / |.| = 1): per candidate pair
# the centre cull; per pair within the cutoff the 16 piece-box tests; per
# piece pair whose boxes overlap the reference's clip + backward of each piece
# against the other and both pose backwards (the average over the seeded
# 8 x n = 200 initial packings, tests/test_bench_contract_cpu.py re-derives
# it); per tree and evaluation its sin / cos, piece boxes and boundary term;
# per history entry element the two-loop recursion, per parameter the rest
# of an lbfgs iteration.  The kernel itself executes fewer operations (one
# boundary assembly gives the area and both gradients), so this is the
# problem's work, not the instructions issued.
FLOPS_PER_PAIR = 6
FLOPS_PER_NEAR = 64
FLOPS_PER_PIECE_PAIR = 1065
FLOPS_PER_TREE = 182 + 338
FLOPS_PER_HIST_ELEM = 10
FLOPS_PER_ITER_ELEM = 16

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one relaxation
# launch, from a one-pass ncu capture of that launch (the mean of two
# launches), per (E, n, iterations, history); other configurations report
# null.  Most of it is written back from L2 while packings run: L-BFGS history
# (2 m (3n + 3) floats per packing; a finished packing's history is discarded
# from L2, not written back) and spilled registers evicted with it.
TRAFFIC_BYTES = {(4096, 200, 200, 10): 87.4e6}
HBM_FALLBACK_GBPS = 6650.0


def measured_hbm_gbps():
    """The measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json
    beside this file), else the earlier measurement on the pool."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return HBM_FALLBACK_GBPS, "fallback"


def reference_lbfgs():
    """The reference's own batched L-BFGS (core/lbfgs_torch_parallel.py:411-729),
    imported unmodified from the reference package that baseline/install_ref.py
    installs into baseline/_ref (torch only).  None when it is not installed."""
    import importlib.util
    path = os.path.join(ROOT, "baseline", "_ref", "core", "lbfgs_torch_parallel.py")
    if not os.path.exists(path):
        return None
    spec = importlib.util.spec_from_file_location("reference_lbfgs_torch_parallel", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.lbfgs


def run_simulation_plain(lbfgs_ref, cost_fn, xyt, h, iters, hist):
    """OptimizerBFGS.run_simulation's flow (pack_dynamics.py:73-137) with torch
    in place of cupy: x = [xyt, h] flattened per packing, an objective that
    unflattens through persistent buffers, evaluates the cost terms and
    flattens the gradients into a fresh array (:95-124), and the reference's
    lbfgs with pack_dynamics' arguments (tolerances 0, no line search).
    cost_fn(xyt, h, cost, grad, grad_h) fills the three outputs."""
    import torch
    E, n = int(xyt.shape[0]), int(xyt.shape[1])
    ns = 3 * n
    x0 = torch.cat([xyt.reshape(E, -1), h], 1).contiguous()
    tmp_x = torch.zeros_like(x0)
    tmp_xyt = xyt.clone()
    tmp_h = h.clone()
    tmp_cost = torch.zeros(E, device=xyt.device)
    tmp_grad = torch.zeros_like(xyt)
    tmp_grad_h = torch.zeros_like(h)

    def f_torch(x, is_main_loop):
        M = x.shape[0]
        tmp_x[:M] = x
        tmp_xyt[:M] = tmp_x[:M, :ns].reshape(M, -1, 3)
        tmp_h[:M] = tmp_x[:M, ns:]
        cost_fn(tmp_xyt[:M], tmp_h[:M], tmp_cost[:M], tmp_grad[:M], tmp_grad_h[:M])
        res = torch.zeros_like(tmp_x[:M])
        res[:, :ns] = tmp_grad[:M].reshape(M, -1)
        res[:, ns:] = tmp_grad_h[:M]
        return tmp_cost[:M], res

    lbfgs_ref(f_torch, x0, tolerance_grad=0, tolerance_change=0, tolerance_rel_change=0.0, max_iter=iters,
              history_size=hist, max_step=0.01, line_search_fn=None, stop_on_cost_increase=False)
    return x0, tmp_cost


def time_plain(torch, dev, lbfgs_ref, cost_fn, xyt, h, iters, hist):
    """One warm-up relaxation of 3 iterations, then one full relaxation timed
    with CUDA events on the current stream (the host loop's syncs included)."""
    run_simulation_plain(lbfgs_ref, cost_fn, xyt, h, 3, hist)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    x, cost = run_simulation_plain(lbfgs_ref, cost_fn, xyt, h, iters, hist)
    e1.record()
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / 1e3, x, cost


def measure_plain_reference(args, dev, xyt, h, spec, fused_value, fused_loss):
    """The plain forms of the north star's comparison, on the same GPU:
    P (plain_reference_lbfgs): this package's cost kernel under the reference's
    unmodified lbfgs, driven as pack_dynamics drives it; R
    (reference_gpu_stack): the reference's own cost kernels, built from its
    source, under the same lbfgs.  R runs on a smaller batch (its area kernel
    takes about 100 ms per evaluation of 4096 packings)."""
    import torch

    from packing_b200.cost import compound_cost
    lbfgs_ref = reference_lbfgs()
    if lbfgs_ref is None:
        why = "reference package not installed in baseline/_ref (python baseline/install_ref.py)"
        return {"unavailable": why}, {"unavailable": why}
    n, iters, hist = args.n, args.iters, args.history

    def ours(x, hh, c, g, gh):
        compound_cost(x, hh, spec, out_cost=c, out_grad=g, out_grad_h=gh)

    Ep = args.plain_E
    dt, _, cost = time_plain(torch, dev, lbfgs_ref, ours, xyt[:Ep], h[:Ep], iters, hist)
    p = {"value": Ep / dt, "unit": "relaxations/s", "E": Ep, "seconds": dt,
         "what": "reference lbfgs (baseline/_ref core/lbfgs_torch_parallel.py, unmodified) driven as "
                 "pack_dynamics.OptimizerBFGS does, over packing_b200.cost.compound_cost",
         "mean_final_loss": float(cost.double().mean()), "fused_mean_final_loss": fused_loss,
         "fused_over_plain_ref": fused_value / (Ep / dt)}
    r = {"unavailable": "reference kernels not built in oracle/_ref (oracle/build_ref.py)"}
    try:
        from oracle import ref_kernels as RK
        if RK.available():
            def reference_kernels(x, hh, c, g, gh):
                cb, gb, _ = RK.boundary(x, hh)
                co, go = RK.overlap(x, False)
                torch.add(cb, co, out=c)
                torch.add(gb, go, out=g)
                gh.zero_()      # use_fixed_h zeroes every term's h gradient (pack_cost.py:178-189)

            Er = args.refgpu_E
            dr, _, _ = time_plain(torch, dev, lbfgs_ref, reference_kernels, xyt[:Er], h[:Er], iters, hist)
            r = {"value": Er / dr, "unit": "relaxations/s", "E": Er, "seconds": dr,
                 "what": "reference lbfgs (unmodified) over the reference's own CUDA kernels "
                         "(multi_overlap_list_total area variant + multi_boundary_distance_list_total, "
                         "pack_cuda.py:482-757) compiled from its source for sm_100a, same GPU",
                 "fused_over_reference_stack": fused_value / (Er / dr)}
    except Exception as exc:   # reported; the headline stands
        r = {"error": f"{type(exc).__name__}: {exc}"}
    return p, r


def measure_c1(args, dev):
    """64 packings of n = 20 (seed 0), overlap-area cost and
    its gradient.  CPU: the FP64 oracle on the host's cores (OpenMP over
    packings), repeated for about 2 s.  GPU: pack_cuda.overlap_multi_ensemble on
    the same FP32 inputs, CUDA-event timed; its error against FP64."""
    import torch

    from oracle import oracle as O
    from packing_b200 import pack_cuda
    E, n = 64, 20
    xyt, _ = workload(E, n, seed=0)
    x64 = xyt.astype(np.float64)
    O.pair_cost(x64, False)
    reps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < 2.0:
        oc, og = O.pair_cost(x64, False)
        reps += 1
    cpu_s = (time.perf_counter() - t0) / reps
    xt = torch.from_numpy(xyt).to(dev)
    c = torch.empty(E, device=dev)
    g = torch.empty_like(xt)
    for _ in range(10):
        pack_cuda.overlap_multi_ensemble(xt, xt, False, out_cost=c, out_grads=g)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = 200
    e0.record()
    for _ in range(k):
        pack_cuda.overlap_multi_ensemble(xt, xt, False, out_cost=c, out_grads=g)
    e1.record()
    torch.cuda.synchronize(dev)
    gpu_s = e0.elapsed_time(e1) / 1e3 / k
    cg, gg = c.double().cpu().numpy(), g.double().cpu().numpy()
    rel = np.abs(cg - oc) / np.maximum(np.abs(oc), 1e-12)
    return {"workload": f"{E} packings x n={n}, seed 0, overlap-area cost + gradient",
            "cpu_evals_per_s": E / cpu_s, "cpu_cores": O.num_threads(), "cpu_kind": "port",
            "cpu_what": "FP64 C restatement of multi_overlap_list_total (area), OpenMP over packings",
            "gpu_evals_per_s": E / gpu_s, "gpu_us_per_call": gpu_s * 1e6,
            "gpu_what": "pack_cuda.overlap_multi_ensemble (pk_overlap), one launch per call, CUDA events",
            "max_cost_rel_err_vs_fp64": float(rel.max()), "max_grad_abs_err_vs_fp64": float(np.abs(gg - og).max()),
            "tolerances": "cost rtol 1e-5, gradient rtol = atol = 1e-4 (pack_test.py:286-297)"}


def run_ours(args, rank, world, dev):
    import torch

    from packing_b200 import _lib
    from packing_b200.cost import CostSpec
    from packing_b200.lbfgs_torch_parallel import lbfgs
    from packing_b200.relax import RelaxParams, relax_into, workspace_floats
    from packing_b200.tune import tuned

    E, n, iters, hist = args.E, args.n, args.iters, args.history
    _lib.ensure_init(dev)
    L = _lib.load()
    xyt_np, h_np = workload(E, n, seed=rank)
    xyt = torch.from_numpy(xyt_np).to(dev)
    h = torch.from_numpy(h_np).to(dev)
    xo = torch.empty_like(xyt)
    ho = torch.empty_like(h)
    loss = torch.empty(E, device=dev)
    iters_out = torch.empty(E, dtype=torch.int32, device=dev)
    work = torch.empty(workspace_floats([n] * E, hist), device=dev)
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)
    # launch shape (threads per packing, persistent grid) from the autotuner;
    # tuning runs before the warm-up and outside the timed region
    prm = RelaxParams(n_iterations=iters, history_size=hist, max_step=0.01, final_eval=False)
    if not args.no_tune:
        prm = tuned(prm, n, spec, dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev)   # > 126 MB L2
    st = torch.cuda.current_stream(dev)

    def launch():
        relax_into(xyt, h, xo, ho, loss, work, spec, prm, iters_out=iters_out)

    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize(dev)
    # one step = one replay of a CUDA graph holding the relaxation launch
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(st)
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            launch()
    st.wait_stream(side)
    graph.replay()
    torch.cuda.synchronize(dev)

    def step():
        graph.replay()

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    clk = ClockSampler(dev.index if rank == 0 else -1)
    if rank == 0:
        clk.start()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        step()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    torch.cuda.synchronize(dev)
    clocks = clk.stop() if rank == 0 else None
    total = sum(times)
    if world > 1:
        t = torch.tensor([total], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total = float(t.item())
        torch.distributed.barrier()
    value = E * world * args.steps / total
    ms_per_step = total / args.steps * 1e3
    kernel_s = total / args.steps
    # an instance stops before max_iter only by the reference's own tests
    # (lbfgs_torch_parallel.py:602-607, 692-724); reported, the work counters
    # below count the iterations actually run
    stopped_early = int((iters_out < iters).sum())
    if not bool(torch.isfinite(loss).all()):
        raise RuntimeError("non-finite loss in the relaxation output")

    out = {"metric": METRIC, "value": value, "unit": "relaxations/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform poses, fixed square side)",
           "config": {"workload": f"batched L-BFGS relaxation, fused one-launch form: E={E} packings x n={n} "
                                  f"trees per GPU, history m={hist}, {iters} iterations, max_step 0.01, "
                                  "cost boundary + overlap area, fixed h",
                      "E_per_gpu": E, "n": n, "history": hist, "iterations": iters,
                      "parallelism": f"instance sharding x{world}", "l2": "flushed between timed steps (256 MB write)",
                      "launch": f"CUDA graph replay of one relaxation launch, {prm.threads or 'default'} threads per "
                                f"packing, {'persistent grid' if prm.persistent else 'one CTA per packing'} "
                                "(autotuned)",
                      "instances_stopped_early": stopped_early},
           "gpu_launches": args.steps, "clocks": clocks}
    if args.quick:
        return out if rank == 0 else None

    # ---- e2e through the public API, pinned host buffers: every rank at once,
    # whole-job value over the slowest rank like the device-timed value ----
    if world > 1:
        torch.distributed.barrier()
    xyt_host = torch.from_numpy(xyt_np).pin_memory()
    h_host = torch.from_numpy(h_np).pin_memory()
    xo_host = torch.empty_like(xyt_host).pin_memory()
    loss_host = torch.empty(E).pin_memory()
    e2e_times = []
    for k in range(args.e2e_steps + 1):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        xd = xyt_host.to(dev, non_blocking=True)
        hd = h_host.to(dev, non_blocking=True)
        relax_into(xd, hd, xo, ho, loss, work, spec, prm)
        xo_host.copy_(xo, non_blocking=True)
        loss_host.copy_(loss, non_blocking=True)
        e1.record(st)
        e1.synchronize()
        if k > 0:
            e2e_times.append(e0.elapsed_time(e1) / 1e3)
    e2e_total = sum(e2e_times)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_total = float(t.item())
        torch.distributed.barrier()
    e2e = E * world * len(e2e_times) / e2e_total
    out["e2e"] = {"value": e2e, "unit": "relaxations/s",
                  "h2d_bytes_per_step": world * (xyt_host.numel() * 4 + h_host.numel() * 4),
                  "d2h_bytes_per_step": world * (xo_host.numel() * 4 + loss_host.numel() * 4)}
    if rank != 0:
        return None

    # ---- roofline: counted work of the same launch, FP32 SIMT peak ----
    counters = torch.zeros(6, dtype=torch.int64, device=dev)
    prm_c = dataclasses.replace(prm, counters=counters)
    relax_into(xyt, h, xo, ho, loss, work, spec, prm_c)
    torch.cuda.synchronize(dev)
    cnt = counters.cpu().numpy().astype(np.float64)
    N = 3 * n + 3
    flops = (cnt[0] * FLOPS_PER_PAIR + cnt[1] * FLOPS_PER_NEAR + cnt[2] * FLOPS_PER_PIECE_PAIR
             + cnt[3] * n * FLOPS_PER_TREE + cnt[5] * FLOPS_PER_HIST_ELEM + cnt[4] * N * FLOPS_PER_ITER_ELEM)
    peak = fp32_peak_tflops(torch, L, dev)
    achieved = flops / kernel_s / 1e12
    traffic = TRAFFIC_BYTES.get((E, n, iters, hist))
    hbm_peak, hbm_src = measured_hbm_gbps()
    out["roofline"] = {"bound": "fp32_simt", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                       "frac": achieved / peak, "traffic": traffic,
                       "peak_source": "measured FP32 FMA probe on this GPU (pk_fma_probe); no tensor-core work: "
                                      "pairwise clipping is not a contraction",
                       "hbm": None if traffic is None else {
                           "achieved_GBps": traffic / kernel_s / 1e9, "peak_GBps": hbm_peak,
                           "frac": traffic / kernel_s / 1e9 / hbm_peak, "peak_source": hbm_src},
                       "work": {"pairs_enumerated": cnt[0], "near_pairs": cnt[1], "piece_pairs": cnt[2],
                                "cost_evals": cnt[3], "iterations": cnt[4], "history_elements": cnt[5],
                                "flops": flops,
                                "flops_per_unit": {"pair": FLOPS_PER_PAIR, "near_pair": FLOPS_PER_NEAR,
                                                   "piece_pair": FLOPS_PER_PIECE_PAIR, "tree_eval": FLOPS_PER_TREE,
                                                   "history_element": FLOPS_PER_HIST_ELEM,
                                                   "parameter_iteration": FLOPS_PER_ITER_ELEM},
                                "counted_on": "the reference's arithmetic (oracle op-counting mode)"}}

    # ---- plain drop-in: the reference-style lbfgs loop over the cost kernel ----
    if not args.skip_plain:
        from packing_b200.cost import compound_cost
        Ep = args.plain_E
        gbuf = torch.empty((Ep, n, 3), device=dev)
        ghbuf = torch.empty((Ep, 3), device=dev)
        cbuf = torch.empty(Ep, device=dev)

        def f(x, is_main):
            compound_cost(x[:, :3 * n].reshape(Ep, n, 3).contiguous(), x[:, 3 * n:].contiguous(), spec,
                          out_cost=cbuf, out_grad=gbuf, out_grad_h=ghbuf)
            return cbuf, torch.cat([gbuf.reshape(Ep, -1), ghbuf], 1)

        x0 = torch.cat([xyt[:Ep].reshape(Ep, -1), h[:Ep]], 1).contiguous()
        x = x0.clone()
        lbfgs(f, x, max_iter=3, history_size=hist, max_step=0.01, tolerance_grad=0, tolerance_change=0)
        torch.cuda.synchronize(dev)
        x = x0.clone()
        t0 = time.perf_counter()
        lbfgs(f, x, max_iter=iters, history_size=hist, max_step=0.01, tolerance_grad=0, tolerance_change=0)
        torch.cuda.synchronize(dev)
        pt = time.perf_counter() - t0
        out["plain_dropin"] = {"value": Ep / pt, "unit": "relaxations/s", "E": Ep,
                               "what": "packing_b200.lbfgs_torch_parallel.lbfgs (per-iteration launches, "
                                       "host loop) over packing_b200.cost.compound_cost",
                               "fused_over_plain": value / (Ep / pt)}

    # ---- the north star's plain forms: the reference's own lbfgs over this
    # package's cost kernel (P) and over the reference's kernels (R) ----
    if not args.skip_ref_legs:
        relax_into(xyt, h, xo, ho, loss, work, spec, prm)
        torch.cuda.synchronize(dev)
        try:
            p, r = measure_plain_reference(args, dev, xyt, h, spec, value, float(loss.double().mean()))
        except Exception as exc:   # reported, the headline stands
            p = r = {"error": f"{type(exc).__name__}: {exc}"}
        out["plain_reference_lbfgs"] = p
        out["reference_gpu_stack"] = r
        if "value" in p:
            out["fused_over_plain_ref"] = value / p["value"]
            out["north_star_10x"] = {"target": 10.0, "fused_over_plain_ref": value / p["value"],
                                     "met": value / p["value"] >= 10.0}
        try:
            out["c1"] = measure_c1(args, dev)
        except Exception as exc:   # reported, the headline stands
            out["c1"] = {"error": f"{type(exc).__name__}: {exc}"}

    # ---- secondary configurations: serving, ragged LUT, GA generation ----
    if not args.skip_extra:
        for name, fn in [("serve", measure_serve), ("ragged_lut", measure_ragged_lut), ("ga_step", measure_ga_step),
                         ("legalize", measure_legalize)]:
            try:
                out[name] = fn(args, dev)
            except Exception as exc:   # reported, the headline stands
                out[name] = {"error": f"{type(exc).__name__}: {exc}"}

    # ---- CPU baseline (oracle, host cores) ----
    if not args.skip_cpu:
        v, cores, dt = cpu_baseline_relax(args.cpu_E, n, iters, hist)
        out["cpu_baseline"] = {"value": v, "unit": "relaxations/s", "cores": cores, "kind": "port",
                               "sample": f"{args.cpu_E} packings x n={n}, {iters} iterations, m={hist} "
                                         f"({dt:.1f} s, FP64 C oracle + numpy lbfgs restatement)"}
    return out


def _serve_requests(count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(10), np.log(200)))))
        xyt, h = workload(1, n, seed=seed * 100003 + k)
        reqs.append((xyt[0], h[0], int(rng.integers(50, 301))))
    return reqs


def measure_serve(args, dev):
    """10,000 requests, n log-uniform in [10, 200], 50-300 iterations, Poisson
    arrivals at ~80% of the measured service capacity (a saturating burst of
    args.serve_burst requests through the pipelined engine); against the
    engine's ceiling on the same mix and the same jobs run batch by batch
    through the plain forms (grouped by tree count and budget, as
    pack_dynamics.run_simulation_list groups by tree count)."""
    import torch

    from packing_b200.cost import CostSpec, compound_cost
    from packing_b200.lbfgs_torch_parallel import lbfgs
    from packing_b200.serve import RelaxServer
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)
    hist = args.history
    # capacity: a saturating burst
    burst = _serve_requests(args.serve_burst, seed=7)
    srv = RelaxServer(spec, history=hist, chunk_iters=args.serve_chunk, device=dev)
    srv.run_trace(burst[:64], np.zeros(64))
    srv = RelaxServer(spec, history=hist, chunk_iters=args.serve_chunk, device=dev)
    cap, _ = srv.run_trace(burst, np.zeros(len(burst)))
    capacity = cap["relaxations_per_s"]
    # Poisson trace at 80 % of capacity
    reqs = _serve_requests(args.serve_requests, seed=11)
    rate = 0.8 * capacity
    arrivals = np.cumsum(np.random.default_rng(12).exponential(1.0 / rate, size=len(reqs)))
    srv = RelaxServer(spec, history=hist, chunk_iters=args.serve_chunk, device=dev)
    stats, done = srv.run_trace(reqs, arrivals)
    # jobs that met the reference's own stop tests before their iteration budget
    stopped_early = sum(1 for r in done if r.iterations < r.iters)
    # the engine's ceiling on the same mix: every burst job resident at once,
    # one step of chunk 300 (so each job runs to its own budget in one launch
    # per size class), device time of the launches only
    srv = RelaxServer(spec, history=hist, chunk_iters=300, device=dev)
    for xyt, h, it in burst[:64]:
        srv.submit(xyt, h, it)
    srv.timed_step()
    srv = RelaxServer(spec, history=hist, chunk_iters=300, device=dev)
    for xyt, h, it in burst:
        srv.submit(xyt, h, it)
    done_c, dev_s = srv.timed_step()
    if len(done_c) != len(burst):
        raise RuntimeError("the ceiling step did not finish every burst job")
    ceiling = len(burst) / dev_s
    # batch-by-batch plain forms on a subset: all requests available, batches
    # of args.serve_plain_batch, one relaxation per distinct (tree count,
    # iteration budget) -- static batching that runs each job to its own
    # budget.  P: the reference's own lbfgs over this package's cost kernel
    # (run_simulation_plain); also this package's drop-in lbfgs.
    def plain_rate(sub, relax_group):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for b0 in range(0, len(sub), args.serve_plain_batch):
            batch = sub[b0:b0 + args.serve_plain_batch]
            groups = {}
            for xyt, h, it in batch:
                groups.setdefault((xyt.shape[0], it), []).append((xyt, h, it))
            for (n, it), grp in groups.items():
                xg = torch.from_numpy(np.stack([g[0] for g in grp])).to(dev)
                hg = torch.from_numpy(np.stack([g[1] for g in grp])).to(dev)
                relax_group(xg, hg, it).cpu()
        return len(sub) / (time.perf_counter() - t0)

    def ours_cost(x, hh, c, g, gh):
        compound_cost(x, hh, spec, out_cost=c, out_grad=g, out_grad_h=gh)

    def dropin_group(xg, hg, it):
        E, n = int(xg.shape[0]), int(xg.shape[1])
        x0 = torch.cat([xg.reshape(E, -1), hg], 1).contiguous()
        cb, gb, ghb = torch.empty(E, device=dev), torch.empty_like(xg), torch.empty_like(hg)

        def f(x, is_main):
            compound_cost(x[:, :3 * n].reshape(E, n, 3).contiguous(), x[:, 3 * n:].contiguous(), spec,
                          out_cost=cb, out_grad=gb, out_grad_h=ghb)
            return cb, torch.cat([gb.reshape(E, -1), ghb], 1)

        return lbfgs(f, x0, max_iter=it, history_size=hist, max_step=0.01, tolerance_grad=0, tolerance_change=0)

    plain_dropin = plain_rate(reqs[:args.serve_plain], dropin_group)
    lbfgs_ref = reference_lbfgs()
    plain_ref = None
    if lbfgs_ref is not None:
        plain_ref = plain_rate(reqs[:args.serve_plain_ref],
                               lambda xg, hg, it: run_simulation_plain(lbfgs_ref, ours_cost, xg, hg, it, hist)[0])
    plain = plain_ref if plain_ref is not None else plain_dropin
    return {"requests": stats["requests"], "arrival_rate_per_s": rate, "capacity_per_s": capacity,
            "ceiling_per_s": ceiling, "capacity_over_ceiling": capacity / ceiling,
            "ceiling_what": f"device time of the same engine's launches with all {len(burst)} burst jobs "
                            "resident and one chunk of 300 iterations (each job to its own budget)",
            "p50_ms": stats["p50_ms"], "p99_ms": stats["p99_ms"], "relaxations_per_s": stats["relaxations_per_s"],
            "engine_launches": stats["launches"], "chunk_iters": args.serve_chunk,
            "plain_batch_by_batch_per_s": plain,
            "plain_what": ("P: the reference's lbfgs (baseline/_ref, unmodified) over packing_b200.cost.compound_cost"
                           if plain_ref is not None else "this package's drop-in lbfgs (reference not installed)"),
            "plain_sample": f"first {args.serve_plain_ref if plain_ref is not None else args.serve_plain} requests, "
                            f"batches of {args.serve_plain_batch}, one relaxation per (n, iteration budget)",
            "plain_dropin_batch_by_batch_per_s": plain_dropin,
            "plain_dropin_sample": f"first {args.serve_plain} requests, this package's drop-in lbfgs",
            "served_over_plain": stats["relaxations_per_s"] / plain, "jobs_stopped_early": stopped_early,
            "workload": "n log-uniform [10,200], iterations U{50..300}, Poisson arrivals at 0.8 x capacity, m="
                        f"{hist}, max_step 0.01, boundary + overlap area"}


def lut_gather_roofline(lookups_per_s, lut, dev):
    """The LUT cost kernel's trilinear lookups per second against the measured
    ceiling of lookups on random cells of the same table."""
    import torch

    from packing_b200 import _lib
    peak = gather_peak(torch, _lib.load(), lut.lut_d, dev)
    return {"achieved_lookups_per_s": lookups_per_s, "peak_lookups_per_s": peak, "frac": lookups_per_s / peak,
            "peak_source": "measured: 8-corner lookups on uniformly random cells of the same table "
                           "(pk_gather_probe)"}


def measure_ragged_lut(args, dev):
    """8192 instances, n log-uniform in [5, 200], LUT 256 x 256 x 360 built
    from the overlap-area kernel; one launch relaxes them all.  The same batch
    is then relaxed on the GA's production fitness cost (pack_ga3.py:1475-1477):
    boundary + the exact-separation LUT (max(0, v)^2) on the reference's
    default 900^3 grid (pack_cost.py:1144-1215), built on the GPU and trimmed."""
    import torch

    from packing_b200 import pack_cuda_lut
    from packing_b200.cost import CostSpec
    from packing_b200.pack_cuda_lut import LookupTable
    from packing_b200.relax import RelaxParams, relax_into, size_classes, workspace_floats
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    X = np.linspace(-2 * 0.5796198, 2 * 0.5796198, 510, dtype=np.float32)[254:]
    Y = np.linspace(-2 * 0.5796198, 2 * 0.5796198, 256, dtype=np.float32)
    T = np.linspace(-np.pi, np.pi, 360, dtype=np.float32)
    lut = LookupTable.build_from_kernel("area", X=X, Y=Y, theta=T, trim_zeros=False, device=dev)
    torch.cuda.synchronize(dev)
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(5)
    E = args.lut_E
    sizes = np.round(np.exp(rng.uniform(np.log(5), np.log(200), size=E))).astype(int)
    xs = [workload(1, int(nn), seed=1000 + k)[0][0] for k, nn in enumerate(sizes)]
    hs = np.concatenate([workload(1, int(nn), seed=0)[1] for nn in sizes])
    flat = torch.from_numpy(np.concatenate(xs)).to(dev)
    off = torch.tensor(np.concatenate([[0], np.cumsum(sizes)]), dtype=torch.int32, device=dev)
    order_h = np.argsort(-sizes, kind="stable")
    order = torch.tensor(order_h, dtype=torch.int32, device=dev)
    classes = size_classes(sizes[order_h])
    h = torch.from_numpy(hs).to(dev)
    prm = RelaxParams(n_iterations=args.iters, history_size=args.history, max_step=0.01, final_eval=False)
    xo = torch.empty_like(flat)
    ho = torch.empty_like(h)
    loss = torch.empty(E, device=dev)
    work = torch.empty(workspace_floats(sizes.tolist(), args.history), device=dev)
    nmax = int(sizes.max())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_relax(spec, cls=classes, reps=3):
        for _ in range(2):
            relax_into(flat, h, xo, ho, loss, work, spec, prm, offsets=off, order=order, n_max=nmax, classes=cls)
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(reps):
            relax_into(flat, h, xo, ho, loss, work, spec, prm, offsets=off, order=order, n_max=nmax, classes=cls)
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / 1e3 / reps

    def time_graph(spec, reps=3):
        # the class launches and their stream fork / join captured once, replayed per step
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            relax_into(flat, h, xo, ho, loss, work, spec, prm, offsets=off, order=order, n_max=nmax, classes=classes)
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            relax_into(flat, h, xo, ho, loss, work, spec, prm, offsets=off, order=order, n_max=nmax, classes=classes)
        g.replay()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        del g
        return e0.elapsed_time(e1) / 1e3 / reps

    area_lut_spec = CostSpec(pair="lut", w_pair=1.0, w_boundary=1.0, w_area=0.0, fixed_h=True, lut=lut)
    relax_s = time_graph(area_lut_spec)
    single_s = time_relax(area_lut_spec, cls=None)

    # the reference's grouping (pack_dynamics.py:177-183): one uniform launch per distinct n, one after another
    groups = {}
    for k, nn in enumerate(sizes):
        groups.setdefault(int(nn), []).append(k)
    gbufs = []
    for nn, ks in groups.items():
        xg = torch.from_numpy(np.stack([xs[k] for k in ks])).to(dev)
        hg = torch.from_numpy(hs[ks]).to(dev)
        gbufs.append((xg, hg, torch.empty_like(xg), torch.empty_like(hg), torch.empty(len(ks), device=dev),
                      torch.empty(workspace_floats([nn] * len(ks), args.history), device=dev)))

    def run_grouped():
        for xg, hg, xgo, hgo, lg, wg in gbufs:
            relax_into(xg, hg, xgo, hgo, lg, wg, area_lut_spec, prm)

    run_grouped()
    torch.cuda.synchronize(dev)
    e0.record()
    run_grouped()
    e1.record()
    torch.cuda.synchronize(dev)
    grouped_s = e0.elapsed_time(e1) / 1e3
    del gbufs
    # LUT cost kernel alone: algorithmic bytes = 8 corners x 4 B per near pair
    cost = torch.empty(E, device=dev)
    grad = torch.empty_like(flat)
    pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(10):
        pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax)
    e1.record()
    torch.cuda.synchronize(dev)
    lut_ms = e0.elapsed_time(e1) / 10
    # and one launch per size class, the form the relaxation above uses
    from packing_b200.classes import ragged_plan
    order_c, classes_c = ragged_plan(sizes.tolist(), dev)
    pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax, order=order_c,
                                                classes=classes_c)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(10):
        pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax, order=order_c,
                                                    classes=classes_c)
    e1.record()
    torch.cuda.synchronize(dev)
    lut_cls_ms = e0.elapsed_time(e1) / 10
    near = 0
    for k in range(0, E, max(1, E // 256)):      # sampled near-pair count
        xk = xs[k]
        dx = xk[:, None, :2] - xk[None, :, :2]
        near += int(((dx ** 2).sum(-1) <= (2 * 0.5796198) ** 2).sum() - len(xk)) // 2
    near_total = near * (E / len(range(0, E, max(1, E // 256))))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    exact = LookupTable.build_exact_separation(device=dev)
    torch.cuda.synchronize(dev)
    exact_build_s = time.perf_counter() - t0
    exact_s = time_graph(CostSpec(pair="lut", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True, lut=exact))
    return {"instances": E, "n_range": [int(sizes.min()), int(sizes.max())], "lut_shape": list(lut.lut_d.shape),
            "lut_build_s": build_s, "relaxations_per_s": E / relax_s, "ms_per_step": relax_s * 1e3,
            "launches": len(classes), "iterations": args.iters,
            "size_classes": [[c.n_max, c.count, c.threads] for c in classes],
            "single_launch_relaxations_per_s": E / single_s,
            "grouped_by_n_relaxations_per_s": E / grouped_s, "grouped_by_n_launches": len(groups),
            "lut_cost_kernel_ms": lut_ms,
            "lut_kernel_algorithmic_GBps": near_total * 32 / (lut_ms * 1e-3) / 1e9,
            "lut_cost_kernel_classes_ms": lut_cls_ms,
            "lut_kernel_classes_algorithmic_GBps": near_total * 32 / (lut_cls_ms * 1e-3) / 1e9,
            "lut_gather_roofline": lut_gather_roofline(near_total / (lut_cls_ms * 1e-3), lut, dev),
            "note": "largest first, one launch per size class (n_max, count, threads per CTA) side by side on "
                    "forked streams, captured once in a CUDA graph and replayed per step; LUT tabulates the "
                    "overlap area",
            "production_exact_lut": {"lut_shape": list(exact.lut_d.shape), "build_s": exact_build_s,
                                     "relaxations_per_s": E / exact_s, "ms_per_step": exact_s * 1e3,
                                     "cost": "GA fitness: boundary + exact-separation LUT (900^3 grid trimmed), "
                                             "max(0, v)^2, fixed h"}}


def measure_ga_step(args, dev):
    """2048 packings of n = 100: Hungarian matching on 100 x 100 costs,
    crossover + Gaussian mutation (0.05, 5 deg), 100-iteration relaxation.
    Then the reference GA's own offspring generation on the same population:
    its default move selector in one launch, and clone + moves + the rough
    relaxation (80 iterations) on its fitness cost with the exact LUT."""
    import torch

    from packing_b200 import lap_batch
    from packing_b200 import pack_move as PM
    from packing_b200.ga_step import (crossover_jitter_step, default_moves, fitness_spec, generation_step,
                                      matching_costs)
    from packing_b200.pack_cuda_lut import LookupTable
    P, n = args.ga_P, 100
    xyt, h = workload(P, n, seed=21)
    pop = torch.from_numpy(xyt).to(dev)
    hh = torch.from_numpy(h).to(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(0)
    partners = torch.randperm(P, generator=gen, device=dev)
    C = matching_costs(pop, pop[partners])
    lap_batch.solve_lap_batch(C)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        lap_batch.solve_lap_batch(C)
    e1.record()
    torch.cuda.synchronize(dev)
    lap_ms = e0.elapsed_time(e1) / 3
    # the reference's diversity metric as a second matrix family (kaggle_support.py:2107-2112)
    mates = pop[partners]
    dd = pop[:, :, None, :2] - mates[:, None, :, :2]
    dt = torch.remainder(pop[:, :, None, 2] - mates[:, None, :, 2] + np.pi, 2 * np.pi) - np.pi
    C2 = torch.sqrt((dd * dd).sum(-1) + dt * dt).to(torch.float32).contiguous()
    del dd, dt
    lap_batch.solve_lap_batch(C2)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(3):
        lap_batch.solve_lap_batch(C2)
    e1.record()
    torch.cuda.synchronize(dev)
    lap2_ms = e0.elapsed_time(e1) / 3
    hbm_peak, hbm_src = measured_hbm_gbps()
    crossover_jitter_step(pop, partners, hh, gen, iterations=args.ga_iters)
    torch.cuda.synchronize(dev)
    e0.record()
    crossover_jitter_step(pop, partners, hh, gen, iterations=args.ga_iters)
    e1.record()
    torch.cuda.synchronize(dev)
    step_ms = e0.elapsed_time(e1)
    # the reference GA's offspring generation
    parents = torch.randint(0, P, (P,), generator=gen, device=dev)
    mates = (parents + torch.randint(1, P, (P,), generator=gen, device=dev)) % P   # never the parent itself
    moves = default_moves()
    mgen = PM.MoveGenerator(seed=5)
    old = PM.Genotype(pop, hh)
    child = PM.Genotype(pop.index_select(0, parents).contiguous(), hh.index_select(0, parents).contiguous())
    rows = torch.arange(P, device=dev)
    entries = [(m[0], m[2]) for m in moves.moves]
    PM.apply_moves(entries, child, rows, old, mates, mgen)
    torch.cuda.synchronize(dev)
    reps = 10
    e0.record()
    for _ in range(reps):
        PM.apply_moves(entries, child, rows, old, mates, mgen, check=False)
    e1.record()
    torch.cuda.synchronize(dev)
    moves_ms = e0.elapsed_time(e1) / reps
    spec = fitness_spec(LookupTable.build_exact_separation(device=dev))
    generation_step(pop, hh, parents, mates, mgen, spec, moves)
    torch.cuda.synchronize(dev)
    e0.record()
    _, _, _, chosen = generation_step(pop, hh, parents, mates, mgen, spec, moves)
    e1.record()
    torch.cuda.synchronize(dev)
    ref_ms = e0.elapsed_time(e1)
    counts = torch.bincount(chosen[chosen >= 0].long(), minlength=len(moves.moves)).cpu().tolist()
    lap_bytes = P * n * n * 4 + P * n * 8
    return {"population": P, "n": n, "lap_instances_per_s": P / (lap_ms * 1e-3), "lap_ms": lap_ms,
            "lap_hbm_GBps": lap_bytes / (lap_ms * 1e-3) / 1e9,
            "lap_hbm_frac": lap_bytes / (lap_ms * 1e-3) / 1e9 / hbm_peak, "lap_hbm_peak_source": hbm_src,
            "lap_reference_metric_ms": lap2_ms,
            "lap_reference_metric": "sqrt(dx^2 + dy^2 + wrap(dtheta)^2), kaggle_support.py:2107-2112",
            "generation_ms": step_ms,
            "generations_per_s": 1e3 / step_ms, "relax_iterations": args.ga_iters,
            "reference_ga_offspring": {
                "moves_ms": moves_ms, "moves_rows_per_s": P / (moves_ms * 1e-3),
                "moves_chosen": dict(zip([m[1] for m in moves.moves], counts)),
                "generation_ms": ref_ms,
                "what": "clone + the GA's default MoveSelector (one pk_moves launch) + 80-iteration rough "
                        "relaxation on boundary + exact-separation LUT, fixed h"}}


def measure_legalize(args, dev):
    """Acceptance of relaxed packings (pack_io.py:28-112): a sample of n = 200
    packings relaxed by the area cost at a looser side, then snapped and
    legalised with the reference's schedule; acceptance is the FP64 legality
    check on the GPU (tests/test_legalize_gpu.py holds it against the
    oracle's independent check)."""
    import torch

    from packing_b200.cost import CostSpec
    from packing_b200.legalize import legalize
    from packing_b200.relax import RelaxParams, relax
    E, n = args.legal_E, args.n
    xyt_np, _ = workload(E, n, seed=31)
    x = torch.from_numpy(xyt_np).to(dev)
    h = torch.zeros((E, 3), device=dev)
    h[:, 0] = float(1.3 * np.sqrt(n * TREE_AREA) + 1.5)
    xr, hr, _, _ = relax(x, h, CostSpec(pair="area", w_area=1e-2, fixed_h=True),
                         RelaxParams(n_iterations=400, history_size=args.history, max_step=0.01))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    r = legalize(xr, hr)
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    legal = r.legal.cpu().numpy()
    side = r.side.cpu().numpy()
    # the FP64 validator alone on the legalised packings tiled to 4096: accepted
    # packings have no overlapping pair, so every near pair runs all its tests
    from packing_b200.validate import validate
    big = r.xyt.repeat(max(1, 4096 // E), 1, 1).contiguous()
    validate(big)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        validate(big)
    e1.record()
    torch.cuda.synchronize(dev)
    vms = e0.elapsed_time(e1) / 5
    validator = {"packings": int(big.shape[0]), "n": n, "ms": vms, "packings_per_s": big.shape[0] / (vms * 1e-3),
                 "what": "pk_validate_fp64 (FP64 side + separating-axis legality) on the legalised packings, "
                         f"tiled {max(1, 4096 // E)}x"}
    return {"packings": E, "n": n, "accepted_fp64": int(legal.sum()), "validator": validator,
            "side_mean_accepted": float(side[legal].mean()) if legal.any() else None,
            "rounds_max": int(r.rounds.max()), "seconds": dt,
            "schedule": "snap, then up to 20 rounds: area weight 1e-2 halved, max_step 1e-4 x sqrt(1/2)^k, "
                        "20000 then 2000 iterations, history 10, until boundary + separation < 1e-10; "
                        "FP64 check; one retry with tolerance_rel_change 0"}


def run_cost_case(args, dev):
    """The compound cost kernel alone (boundary + overlap area and their
    gradients) on E packings of n trees: --steps launches at the seeded
    initial poses, then --steps at the poses after --iters iterations of the
    fused relaxation.  A profiling case, not a benchmark metric."""
    import torch

    from packing_b200 import _lib
    from packing_b200.cost import CostSpec, compound_cost
    from packing_b200.relax import RelaxParams, relax
    _lib.ensure_init(dev)
    E, n = args.E, args.n
    xyt_np, h_np = workload(E, n, seed=0)
    xyt = torch.from_numpy(xyt_np).to(dev)
    h = torch.from_numpy(h_np).to(dev)
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)
    xr, _, _, _ = relax(xyt, h, spec, RelaxParams(n_iterations=args.iters, history_size=args.history,
                                                  max_step=0.01, final_eval=False))
    c = torch.empty(E, device=dev)
    g = torch.empty_like(xyt)
    gh = torch.empty_like(h)
    out = {"case": "cost", "E": E, "n": n}
    for name, x in (("initial", xyt), ("relaxed", xr)):
        for _ in range(args.warmup):
            compound_cost(x, h, spec, out_cost=c, out_grad=g, out_grad_h=gh)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            compound_cost(x, h, spec, out_cost=c, out_grad=g, out_grad_h=gh)
        e1.record()
        torch.cuda.synchronize(dev)
        out[f"ms_{name}"] = e0.elapsed_time(e1) / args.steps
    return out


def run_lut_case(args, dev):
    """The LUT cost kernel alone (pk_overlap_lut, ragged) on the C4 batch:
    --lut-E packings with n log-uniform in [5, 200], LUT 256 x 256 x 360 built
    from the overlap-area kernel: --warmup then --steps launches.  Algorithmic
    bytes: 8 corners x 4 B per near pair.  A profiling case, not a benchmark
    metric."""
    import torch

    from packing_b200 import pack_cuda_lut
    from packing_b200.pack_cuda_lut import LookupTable
    X = np.linspace(-2 * 0.5796198, 2 * 0.5796198, 510, dtype=np.float32)[254:]
    Y = np.linspace(-2 * 0.5796198, 2 * 0.5796198, 256, dtype=np.float32)
    T = np.linspace(-np.pi, np.pi, 360, dtype=np.float32)
    lut = LookupTable.build_from_kernel("area", X=X, Y=Y, theta=T, trim_zeros=False, device=dev)
    rng = np.random.default_rng(5)
    if args.lut_uniform:   # --E packings of --n trees instead of the C4 batch
        E = args.E
        sizes = np.full(E, args.n)
        xs = list(workload(E, args.n, seed=0)[0])
    else:
        E = args.lut_E
        sizes = np.round(np.exp(rng.uniform(np.log(5), np.log(200), size=E))).astype(int)
        xs = [workload(1, int(nn), seed=1000 + k)[0][0] for k, nn in enumerate(sizes)]
    flat = torch.from_numpy(np.concatenate(xs)).to(dev)
    off = torch.tensor(np.concatenate([[0], np.cumsum(sizes)]), dtype=torch.int32, device=dev)
    nmax = int(sizes.max())
    cost = torch.empty(E, device=dev)
    grad = torch.empty_like(flat)
    for _ in range(args.warmup):
        pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    from packing_b200.classes import ragged_plan
    order, classes = ragged_plan(sizes.tolist(), dev)
    for _ in range(args.warmup):
        pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax, order=order,
                                                    classes=classes)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(args.steps):
        pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, cost, lut, grad, n_max=nmax, order=order,
                                                    classes=classes)
    e1.record()
    torch.cuda.synchronize(dev)
    ms_cls = e0.elapsed_time(e1) / args.steps
    near = 0
    for x in xs:
        d = x[:, None, :2] - x[None, :, :2]
        near += int(((d ** 2).sum(-1) <= (2 * 0.5796198) ** 2).sum() - len(x)) // 2
    return {"case": "lut", "instances": E, "lut_shape": list(lut.lut_d.shape), "ms_per_launch": ms,
            "near_pairs": near, "lookups_per_s": near / (ms * 1e-3),
            "gather_roofline": lut_gather_roofline(near / (ms_cls * 1e-3), lut, dev),
            "algorithmic_GBps": near * 32 / (ms * 1e-3) / 1e9, "checksum": float(cost.double().sum()),
            "size_classes": {"ms": ms_cls, "launches": len(classes), "lookups_per_s": near / (ms_cls * 1e-3),
                             "algorithmic_GBps": near * 32 / (ms_cls * 1e-3) / 1e9}}


def run_exact_lut_case(args, dev):
    """The exact-separation table build (pk_lut_build_exact_sep) on the
    reference's default grid of --lut-n points per axis, untrimmed: --warmup
    then --steps builds.  Algorithmic bytes: the float32 table written once.
    A profiling case, not a benchmark metric."""
    import torch

    from packing_b200.pack_cuda_lut import LookupTable
    N = args.lut_n
    X, Y, T = LookupTable.default_grid(N, N, N)
    for _ in range(args.warmup):
        lut = LookupTable.build_exact_separation(X=X, Y=Y, theta=T, trim_zeros=False, device=dev)
        del lut
    torch.cuda.synchronize(dev)
    t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        lut = LookupTable.build_exact_separation(X=X, Y=Y, theta=T, trim_zeros=False, device=dev)
        torch.cuda.synchronize(dev)
        t.append(time.perf_counter() - t0)
        del lut
    ms = 1e3 * min(t)
    bytes_out = 4.0 * len(X) * len(Y) * len(T)
    return {"case": "exact_lut", "grid": [len(X), len(Y), len(T)], "ms_per_build": ms,
            "points_per_s": len(X) * len(Y) * len(T) / (ms * 1e-3), "table_write_GBps": bytes_out / (ms * 1e-3) / 1e9}


def run_moves_case(args, dev):
    """The GA's default move selector (pk_moves) on --ga-P clones of n = --n
    packings, mates from the parent population: --warmup then --steps
    launches timed with CUDA events.  Algorithmic bytes per row: the row read
    and written (24 n B) plus the mate read (12 n B) for crossover rows.  A
    profiling case, not a benchmark metric."""
    import torch

    from packing_b200 import pack_move as PM
    from packing_b200.ga_step import default_moves
    P, n = args.ga_P, args.n
    xyt, h = workload(P, n, seed=21)
    pop = torch.from_numpy(xyt).to(dev)
    hh = torch.from_numpy(h).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    parents = torch.randint(0, P, (P,), generator=g, device=dev)
    mates = (parents + torch.randint(1, P, (P,), generator=g, device=dev)) % P
    old = PM.Genotype(pop, hh)
    child = PM.Genotype(pop.index_select(0, parents).contiguous(), hh.index_select(0, parents).contiguous())
    rows = torch.arange(P, device=dev)
    moves = default_moves()
    entries = [(m[0], m[2]) for m in moves.moves]
    mgen = PM.MoveGenerator(seed=5)
    chosen = PM.apply_moves(entries, child, rows, old, mates, mgen)
    for _ in range(args.warmup):
        PM.apply_moves(entries, child, rows, old, mates, mgen, check=False)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        PM.apply_moves(entries, child, rows, old, mates, mgen, check=False)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    cross = int(((chosen == 7) | (chosen == 8)).sum())
    algo = P * 24.0 * n + cross * 12.0 * n
    return {"case": "moves", "rows": P, "n": n, "ms_per_launch": ms, "rows_per_s": P / (ms * 1e-3),
            "algorithmic_GBps": algo / (ms * 1e-3) / 1e9}


def run_lap_case(args, dev):
    """Batched Hungarian on --ga-P matrices of n = --n trees: squared centre
    distance + |wrapped angle difference| between seeded packings and
    shuffled partners, as the matched crossover builds them; --warmup then
    --steps solves timed with CUDA events.  Algorithmic bytes: the matrices
    read once plus the row matches and totals written.  A profiling case, not
    a benchmark metric."""
    import torch

    from packing_b200 import lap_batch
    from packing_b200.ga_step import matching_costs
    P, n = args.ga_P, args.n
    xyt, _ = workload(P, n, seed=21)
    pop = torch.from_numpy(xyt).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    C = matching_costs(pop, pop[torch.randperm(P, generator=g, device=dev)])
    for _ in range(args.warmup):
        lap_batch.solve_lap_batch(C)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        lap_batch.solve_lap_batch(C)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    algo = P * n * n * 4.0 + P * n * 4.0 + P * 4.0
    return {"case": "lap", "problems": P, "n": n, "ms_per_solve": ms, "problems_per_s": P / (ms * 1e-3),
            "algorithmic_GBps": algo / (ms * 1e-3) / 1e9}


def run_ragged_sharded(args, rank, world, dev):
    """--ragged: one seeded ragged population of args.E x world packings (n
    log-uniform in [5, 200], the C4 size mix, boundary + overlap area),
    partitioned across ranks into contiguous work-balanced ranges
    (shard.partition, work ~ n^2); each rank relaxes its range in one CUDA
    graph of size-class launches, no collective in the timed region; then the
    one per-generation exchange (an all_gather of per-packing loss / side /
    iterations) outside it.  value = all packings / max-over-ranks time."""
    import torch

    from packing_b200 import _lib
    from packing_b200.cost import CostSpec
    from packing_b200.relax import RelaxParams, relax_into, workspace_floats
    from packing_b200.classes import size_classes
    from packing_b200.shard import gather_results, partition
    _lib.ensure_init(dev)
    total = args.E * world
    rng = np.random.default_rng(0)
    sizes = np.round(np.exp(rng.uniform(np.log(5), np.log(200), size=total))).astype(int)
    ranges = partition(sizes, world)
    s0, s1 = ranges[rank]
    mine = sizes[s0:s1]
    xs = [workload(1, int(nn), seed=1000 + k)[0][0] for k, nn in zip(range(s0, s1), mine)]
    hs = np.concatenate([workload(1, int(nn), seed=0)[1] for nn in mine]) if len(mine) else np.zeros((0, 3), np.float32)
    E = len(mine)
    flat = torch.from_numpy(np.concatenate(xs) if E else np.zeros((0, 3), np.float32)).to(dev)
    off = torch.tensor(np.concatenate([[0], np.cumsum(mine)]), dtype=torch.int32, device=dev)
    order_h = np.argsort(-mine, kind="stable")
    order = torch.tensor(order_h, dtype=torch.int32, device=dev)
    classes = size_classes(mine[order_h]) if E else []
    h = torch.from_numpy(hs).to(dev)
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)
    prm = RelaxParams(n_iterations=args.iters, history_size=args.history, max_step=0.01, final_eval=False)
    xo, ho = torch.empty_like(flat), torch.empty_like(h)
    loss = torch.empty(E, device=dev)
    iters_out = torch.empty(E, dtype=torch.int32, device=dev)
    work = torch.empty(max(1, workspace_floats(mine.tolist(), args.history)), device=dev)
    nmax = int(mine.max()) if E else 0

    def launch():
        if E:
            relax_into(flat, h, xo, ho, loss, work, spec, prm, offsets=off, order=order, n_max=nmax,
                       iters_out=iters_out, classes=classes)

    st = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize(dev)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(st)
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            launch()
    st.wait_stream(side)
    torch.cuda.synchronize(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    clk = ClockSampler(dev.index if rank == 0 else -1)
    if rank == 0:
        clk.start()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        graph.replay()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    torch.cuda.synchronize(dev)
    clocks = clk.stop() if rank == 0 else None
    tot = sum(times)
    if world > 1:
        t = torch.tensor([tot], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        tot = float(t.item())
    # the per-generation exchange, outside the timed region
    local = torch.stack([loss.double(), ho[:, 0].double(), iters_out.double()], 1)
    table = gather_results(local, [b - a for a, b in ranges]) if world > 1 else local
    del graph
    if world > 1:
        torch.distributed.barrier()
    if rank != 0:
        return None
    work_share = [float((sizes[a:b].astype(float) ** 2).sum()) for a, b in ranges]
    return {"metric": METRIC, "value": total * args.steps / tot, "unit": "relaxations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ragged population, fixed square sides)",
            "config": {"workload": f"ragged population of {total} packings (n log-uniform [5, 200]), history m="
                                   f"{args.history}, {args.iters} iterations, boundary + overlap area, fixed h; "
                                   f"partitioned into {world} work-balanced contiguous ranges",
                       "E_total": total, "parallelism": f"instance sharding x{world} (shard.partition)",
                       "ranges": ranges, "work_share_max_over_mean": max(work_share) / (sum(work_share) / world),
                       "l2": "flushed between timed steps (256 MB write)",
                       "launch": "CUDA graph replay of the size-class launches"},
            "gathered_rows": int(table.shape[0]), "gpu_launches": args.steps * len(classes), "clocks": clocks}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from oracle import oracle as O
    O.lib()
    vals = []
    for k in range(args.warmup + args.steps):
        v, cores, dt = cpu_baseline_relax(args.ref_E, args.n, args.iters, args.history, seed=1000 + k)
        if k >= args.warmup:
            vals.append((v, dt))
    tot_t = sum(dt for _, dt in vals)
    value = args.ref_E * len(vals) / tot_t
    sample = (f"{args.ref_E} packings x n={args.n} per step, {args.iters} iterations, m={args.history}: FP64 C "
              "restatement of the reference cost kernels + numpy restatement of its lbfgs, OpenMP over packings")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "relaxations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_t / len(vals) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded uniform poses, fixed square side)",
            "config": {"workload": f"batched L-BFGS relaxation, n={args.n}, m={args.history}, {args.iters} iterations "
                                   "(CPU sample of the per-GPU population)", "n": args.n},
            "cpu_baseline": {"value": value, "unit": "relaxations/s", "cores": O.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "relaxations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--E", type=int, default=4096)
    ap.add_argument("--n", type=int, default=200)
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--history", type=int, default=10)
    ap.add_argument("--e2e-steps", dest="e2e_steps", type=int, default=2)
    ap.add_argument("--plain-E", dest="plain_E", type=int, default=4096)
    ap.add_argument("--cpu-E", dest="cpu_E", type=int, default=128)
    ap.add_argument("--ref-E", dest="ref_E", type=int, default=64)
    ap.add_argument("--refgpu-E", dest="refgpu_E", type=int, default=1024,
                    help="packings of the reference-kernel stack leg (R)")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-ref-legs", dest="skip_ref_legs", action="store_true",
                    help="skip the reference-lbfgs plain forms (P, R) and the C1 block")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-extra", action="store_true", help="skip serving / ragged LUT / GA step")
    ap.add_argument("--serve-requests", dest="serve_requests", type=int, default=10000)
    ap.add_argument("--serve-burst", dest="serve_burst", type=int, default=2000)
    ap.add_argument("--serve-chunk", dest="serve_chunk", type=int, default=25)
    ap.add_argument("--serve-plain", dest="serve_plain", type=int, default=128)
    ap.add_argument("--serve-plain-ref", dest="serve_plain_ref", type=int, default=32)
    ap.add_argument("--serve-plain-batch", dest="serve_plain_batch", type=int, default=128)
    ap.add_argument("--lut-E", dest="lut_E", type=int, default=8192)
    ap.add_argument("--ga-P", dest="ga_P", type=int, default=2048)
    ap.add_argument("--ga-iters", dest="ga_iters", type=int, default=100)
    ap.add_argument("--legal-E", dest="legal_E", type=int, default=64)
    ap.add_argument("--quick", action="store_true", help="headline timing only")
    ap.add_argument("--ragged", action="store_true",
                    help="one seeded ragged population of E x gpus packings partitioned across the ranks "
                         "(shard.partition) instead of E uniform packings per rank")
    ap.add_argument("--no-tune", dest="no_tune", action="store_true",
                    help="default launch shape instead of the autotuned one (profiling captures)")
    ap.add_argument("--case", default="relax", choices=["relax", "cost", "exact_lut", "moves", "lut", "lap"],
                    help="relax: the headline; cost: the compound cost kernel alone on E packings, at the "
                         "initial poses and after --iters iterations of relaxation; exact_lut: the exact-separation "
                         "table build on --lut-n points per axis; lut: the LUT cost kernel alone on the C4 batch; "
                         "moves: the GA's move selector on --ga-P rows of --n trees; lap: the batched Hungarian on "
                         "--ga-P matched-crossover matrices of --n trees (profiling captures)")
    ap.add_argument("--lut-n", dest="lut_n", type=int, default=900)
    ap.add_argument("--lut-uniform", dest="lut_uniform", action="store_true",
                    help="--case lut on --E packings of --n trees instead of the C4 batch")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # CPU-only arm: rank 0 measures, the other ranks exit without work
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=dev)
    cases = {"cost": run_cost_case, "exact_lut": run_exact_lut_case, "moves": run_moves_case, "lut": run_lut_case,
             "lap": run_lap_case}
    if args.case in cases:
        out = cases[args.case](args, dev)
    elif args.ragged:
        out = run_ragged_sharded(args, rank, world, dev)
    else:
        out = run_ours(args, rank, world, dev)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
