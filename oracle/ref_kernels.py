"""Launcher for the reference's own CUDA kernels -- TEST INFRASTRUCTURE ONLY.

Loads the cubins that oracle/build_ref.py compiles from the reference source
(core/pack_cuda.py, core/pack_cuda_lut.py, core/lap_batch.py) through the CUDA
driver API into torch's current context, sets their __constant__ tables the
way the reference's host code does (pack_cuda.py:1010-1030,
pack_cuda_lut.py:653-695) and launches them with the reference's grid and
block shapes (pack_cuda.py:1146-1183, 1274-1295; pack_cuda_lut.py:835-862;
lap_batch.py:507-532).  Tests use it to compare this package with the
reference kernels on the same inputs.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_cuda = None
_mods = {}


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f + ".cubin"))
               for f in ("pack_cuda_area", "pack_cuda_sep", "pack_cuda_lut", "lap_batch"))


def _drv():
    global _cuda
    if _cuda is None:
        L = ctypes.CDLL("libcuda.so.1")
        L.cuModuleLoadData.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
        L.cuModuleGetFunction.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_char_p]
        L.cuModuleGetGlobal_v2.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_size_t),
                                           ctypes.c_void_p, ctypes.c_char_p]
        L.cuMemcpyHtoD_v2.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t]
        L.cuLaunchKernel.argtypes = [ctypes.c_void_p] + [ctypes.c_uint] * 7 + [ctypes.c_void_p,
                                                                               ctypes.POINTER(ctypes.c_void_p),
                                                                               ctypes.c_void_p]
        L.cuFuncSetAttribute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        _cuda = L
    return _cuda


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: CUDA driver error {rc}")


def _set_global(mod, name, arr: np.ndarray):
    L = _drv()
    ptr = ctypes.c_uint64()
    size = ctypes.c_size_t()
    _check(L.cuModuleGetGlobal_v2(ctypes.byref(ptr), ctypes.byref(size), mod, name.encode()), f"global {name}")
    data = np.ascontiguousarray(arr)
    assert data.nbytes <= size.value, (name, data.nbytes, size.value)
    _check(L.cuMemcpyHtoD_v2(ptr.value, data.ctypes.data, data.nbytes), f"set {name}")


def _module(name):
    if name in _mods:
        return _mods[name]
    torch.cuda.init()
    torch.zeros(1, device="cuda")   # make torch's primary context current
    L = _drv()
    blob = open(os.path.join(REF_DIR, name + ".cubin"), "rb").read()
    mod = ctypes.c_void_p()
    buf = ctypes.create_string_buffer(blob, len(blob))
    _check(L.cuModuleLoadData(ctypes.byref(mod), buf), f"load {name}")
    if name.startswith("pack_cuda_") and name != "pack_cuda_lut":
        pxy, pnv, txy, R, cut, area = O.geometry()
        _set_global(mod, "const_piece_xy", pxy.astype(np.float32).reshape(-1))
        _set_global(mod, "const_piece_nverts", pnv.astype(np.int32))
        tv = np.zeros(256, np.float32)
        tv[:30] = txy.astype(np.float32).reshape(-1)
        _set_global(mod, "const_tree_vertices_xy", tv)
        _set_global(mod, "const_n_tree_vertices", np.array([15], np.int32))
    _mods[name] = (mod, buf)
    return _mods[name]


def _func(modname, fname):
    mod, _ = _module(modname)
    f = ctypes.c_void_p()
    _check(_drv().cuModuleGetFunction(ctypes.byref(f), mod, fname.encode()), f"function {fname}")
    return f


def _launch(f, grid, block, smem, args):
    """args: list of ctypes values (c_void_p for pointers, c_int, ...)."""
    holders = [a if isinstance(a, ctypes._SimpleCData) else ctypes.c_void_p(a) for a in args]
    params = (ctypes.c_void_p * len(holders))(*[ctypes.cast(ctypes.byref(h), ctypes.c_void_p) for h in holders])
    st = torch.cuda.current_stream().cuda_stream
    _check(_drv().cuLaunchKernel(f, grid, 1, 1, block, 1, 1, smem, ctypes.c_void_p(st), params, None), "launch")


def _p(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def overlap(xyt: torch.Tensor, use_separation: bool, grad: bool = True):
    """multi_overlap_list_total (pack_cuda.py:482): grid E, block 2n."""
    E, n, _ = xyt.shape
    cost = torch.zeros(E, device=xyt.device)
    g = torch.zeros_like(xyt) if grad else None
    f = _func("pack_cuda_sep" if use_separation else "pack_cuda_area", "multi_overlap_list_total")
    _launch(f, E, 2 * n, 0, [_p(xyt), _p(xyt), ctypes.c_int(n), _p(cost), _p(g), ctypes.c_int(E),
                             ctypes.c_int(int(use_separation)), ctypes.c_int(0), ctypes.c_void_p(0),
                             ctypes.c_int(0), ctypes.c_int(2)])
    return cost, g


def boundary(xyt: torch.Tensor, h: torch.Tensor):
    """multi_boundary_distance_list_total (pack_cuda.py:706): grid E, block n."""
    E, n, _ = xyt.shape
    cost = torch.zeros(E, device=xyt.device)
    g = torch.zeros_like(xyt)
    gh = torch.zeros_like(h)
    f = _func("pack_cuda_area", "multi_boundary_distance_list_total")
    _launch(f, E, n, 0, [_p(xyt), ctypes.c_int(n), _p(h), _p(cost), _p(g), _p(gh), ctypes.c_int(E)])
    return cost, g, gh


def lut_overlap(xyt: torch.Tensor, vals: torch.Tensor, bounds, quad: bool):
    """multi_overlap_lut_total (pack_cuda_lut.py:596): grid E, block n,
    12 n bytes of shared memory; the LUT pointer global is set by the host
    before the launch so no block can read it unset."""
    E, n, _ = xyt.shape
    mod, _ = _module("pack_cuda_lut")
    nx, ny, nt = vals.shape
    x0, x1, y0, y1, t0, t1 = [np.float32(b) for b in bounds]
    for name, v in [("c_N_x", np.int32(nx)), ("c_N_y", np.int32(ny)), ("c_N_theta", np.int32(nt)),
                    ("c_X_min", x0), ("c_X_max", x1), ("c_Y_min", y0), ("c_Y_max", y1),
                    ("c_theta_min", t0), ("c_theta_max", t1),
                    ("c_grid_dx", np.float32((x1 - x0) / (nx - 1))), ("c_grid_dy", np.float32((y1 - y0) / (ny - 1))),
                    ("c_grid_dtheta", np.float32((t1 - t0) / (nt - 1))),
                    ("c_apply_quadratic_transform", np.int32(int(quad)))]:
        _set_global(mod, name, np.array([v]))
    _set_global(mod, "g_lut", np.array([vals.data_ptr()], np.uint64))
    cost = torch.zeros(E, device=xyt.device)
    g = torch.zeros_like(xyt)
    f = _func("pack_cuda_lut", "multi_overlap_lut_total")
    _launch(f, E, n, 12 * n, [_p(xyt), ctypes.c_int(n), _p(vals), _p(cost), _p(g), ctypes.c_int(E)])
    return cost, g


def hungarian(C: torch.Tensor):
    """hungarian_kernel + compute_costs (lap_batch.py:62-196, 507-532)."""
    B, N, _ = C.shape
    assert N <= 200, "the reference kernel keeps 200-entry stack arrays (lap_batch.py:100-102)"
    work = torch.empty_like(C)
    rm = torch.full((B, N), -1, dtype=torch.int32, device=C.device)
    cm = torch.full((B, N), -1, dtype=torch.int32, device=C.device)
    u = torch.zeros((B, N), device=C.device)
    v = torch.zeros((B, N), device=C.device)
    tot = torch.empty(B, device=C.device)
    _launch(_func("lap_batch", "hungarian_kernel"), B, 1, 0,
            [_p(C), _p(work), _p(rm), _p(cm), _p(u), _p(v), ctypes.c_int(B), ctypes.c_int(N)])
    _launch(_func("lap_batch", "compute_costs"), (B + 255) // 256, 256, 0,
            [_p(C), _p(rm), _p(tot), ctypes.c_int(B), ctypes.c_int(N)])
    return rm, tot
