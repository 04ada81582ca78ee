"""ctypes binding of libpackb200.so and the tensor plumbing shared by the
drop-in modules.

The library is the product: there is no CPU or torch fallback.  If the
shared object is missing or a CUDA device is absent, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

from . import build as _build

_lock = threading.Lock()
_lib = None
_inited_devices: set[int] = set()

PK_PAIR_NONE, PK_PAIR_AREA, PK_PAIR_SEP, PK_PAIR_LUT = 0, 1, 2, 3
PK_MAX_TREES = 1024
PK_MAX_LAP_N = 256


class PkGeometry(ctypes.Structure):
    _fields_ = [
        ("piece_xy", ctypes.c_double * 2 * 4 * 4),
        ("piece_nv", ctypes.c_int * 4),
        ("tree_xy", ctypes.c_double * 2 * 16),
        ("n_tree_verts", ctypes.c_int),
        ("max_radius", ctypes.c_double),
        ("area", ctypes.c_double),
        ("has_legal", ctypes.c_int),
        ("legal_piece_xy", ctypes.c_double * 2 * 4 * 4),
        ("legal_tree_xy", ctypes.c_double * 2 * 16),
    ]


class PkLut(ctypes.Structure):
    _fields_ = [
        ("vals", ctypes.c_void_p),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nt", ctypes.c_int),
        ("x_min", ctypes.c_float), ("x_max", ctypes.c_float),
        ("y_min", ctypes.c_float), ("y_max", ctypes.c_float),
        ("t_min", ctypes.c_float), ("t_max", ctypes.c_float),
        ("quadratic", ctypes.c_int),
    ]


class PkCostSpec(ctypes.Structure):
    _fields_ = [
        ("pair_mode", ctypes.c_int),
        ("w_pair", ctypes.c_float),
        ("w_boundary", ctypes.c_float),
        ("w_area", ctypes.c_float),
        ("fixed_h", ctypes.c_int),
        ("lut", PkLut),
        ("symmetry", ctypes.c_int),
    ]


class PkRelaxParams(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int), ("history", ctypes.c_int), ("lr", ctypes.c_float),
        ("max_step", ctypes.c_float), ("has_max_step", ctypes.c_int), ("tol_grad", ctypes.c_float),
        ("tol_change", ctypes.c_float), ("tol_rel_change", ctypes.c_float),
        ("stop_on_cost_increase", ctypes.c_int), ("max_eval", ctypes.c_int), ("final_eval", ctypes.c_int),
        ("counters", ctypes.c_void_p),
        ("threads", ctypes.c_int), ("persistent", ctypes.c_int),
    ]


class PkJob(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("max_iter", ctypes.c_int),
        ("x_off", ctypes.c_longlong), ("h_off", ctypes.c_longlong),
        ("status", ctypes.c_int), ("it", ctypes.c_int), ("evals", ctypes.c_int),
        ("hlen", ctypes.c_int), ("hstart", ctypes.c_int),
        ("H", ctypes.c_float), ("loss", ctypes.c_float), ("loss0", ctypes.c_float),
    ]


PK_JOB_NEW, PK_JOB_RUNNING, PK_JOB_DONE = 0, 1, 2


PK_MAX_MOVE_TYPES = 16


class PkMove(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int), ("respect_edge_spacer_filter", ctypes.c_int),
        ("max_xy_move", ctypes.c_double), ("max_theta_move", ctypes.c_double),
        ("min_n_trees", ctypes.c_int), ("max_n_trees", ctypes.c_int),
        ("max_n_trees_ratio", ctypes.c_double),
        ("min_radius", ctypes.c_double), ("max_radius", ctypes.c_double),
        ("simple_mate_location", ctypes.c_int), ("distance_function", ctypes.c_int),
        ("decouple_mate_location", ctypes.c_int), ("use_edge_clearance_when_decoupled", ctypes.c_int),
        ("do_90_rotation", ctypes.c_int),
    ]


class PkGenotype(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("mate_kind", ctypes.c_int), ("filter", ctypes.c_int), ("spacer", ctypes.c_int),
        ("margin", ctypes.c_double), ("dist_x", ctypes.c_double), ("dist_y", ctypes.c_double),
        ("dist_corner", ctypes.c_double),
    ]


class PkMoveSet(ctypes.Structure):
    _fields_ = [
        ("n_moves", ctypes.c_int), ("cum_prob", ctypes.c_double * PK_MAX_MOVE_TYPES),
        ("moves", PkMove * PK_MAX_MOVE_TYPES), ("geno", PkGenotype),
    ]


# (name, argtypes) of every exported entry point; include/packb200.h is the
# authoritative declaration.
_P, _I, _F, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
SIGNATURES = {
    "pk_version": [],
    "pk_default_geometry": [_D, ctypes.POINTER(PkGeometry)],
    "pk_init": [ctypes.POINTER(PkGeometry)],
    "pk_last_error": [],
    "pk_cost": [_P, _P, _I, _I, _P, ctypes.POINTER(PkCostSpec), _P, _P, _P, _P],
    "pk_cost_ordered": [_P, _P, _P, _I, _I, _I, _P, ctypes.POINTER(PkCostSpec), _I, _P, _P, _P, _P],
    "pk_overlap": [_P, _I, _I, _I, _P, _P, _P],
    "pk_overlap_crystal": [_P, _I, _I, _I, _P, _I, _I, _P, _P, _P],
    "pk_boundary": [_P, _P, _I, _I, _P, _P, _P, _P],
    "pk_overlap_lut": [_P, _P, _I, _I, ctypes.POINTER(PkLut), _P, _P, _P],
    "pk_lut_build": [_P, _I, _P, _I, _P, _I, _I, _P, _P],
    "pk_lut_build_exact_sep": [_P, _I, _P, _I, _P, _I, _P, _P],
    "pk_moves": [_P, _P, _I, _I, _P, _I, _P, _P, _I, _P, ctypes.POINTER(PkMoveSet), ctypes.c_uint64, ctypes.c_uint64,
                 _P, _P, _P],
    "pk_move_draws": [ctypes.c_uint64, ctypes.c_uint64, _I, _I, _I, _P, _P],
    "pk_lap_solve": [_P, _I, _I, _P, _P, _P, _P],
    "pk_diversity_matrix": [_P, _P, _I, _I, _I, _I, _P, _P],
    "pk_diversity_costs": [_P, _P, _I, _I, _I, _I, _P, _P],
    "pk_diversity_shortcut": [_P, _P, _I, _I, _I, _F, _F, _I, _P, _P],
    "pk_lbfgs_phase": [_I, _I, _P, _I, _I, _I, _I, _D, _D, _D, _D, _I, _I, _P],
    "pk_wolfe_phase": [_I, _I, _P, _I, _I, _I, _D, _D, _D, _I, _P],
    "pk_wolfe_apply": [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _P],
    "pk_relax": [_P, _P, _P, _P, _I, _I, ctypes.POINTER(PkCostSpec), ctypes.POINTER(PkRelaxParams), _P, _P, _P,
                 _P, _P, _P],
    "pk_relax_ordered": [_P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(PkCostSpec), ctypes.POINTER(PkRelaxParams), _P,
                         _P, _P, _P, _P, _P],
    "pk_relax_workspace_floats": [_P, _I, _I, _I],
    "pk_fma_probe": [_P, _I, _I, _I, _P],
    "pk_gather_probe": [_P, _I, _I, _I, _P, _I, _I, _I, ctypes.c_uint, _P],
    "pk_validate_fp64": [_P, _I, _I, _I, _P, _P, _P],
    "pk_snap": [_P, _P, _I, _I, _P, _P, _P],
    "pk_relax_jobs": [_P, _P, _I, _P, _I, ctypes.POINTER(PkCostSpec), ctypes.POINTER(PkRelaxParams), _I, _P],
    "pk_relax_noalloc": [_P, _P, _I, _I, ctypes.POINTER(PkCostSpec), ctypes.POINTER(PkRelaxParams), _P, _P, _P, _P,
                         _P],
}
RESTYPES = {"pk_last_error": ctypes.c_char_p, "pk_relax_workspace_floats": ctypes.c_size_t}


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load (building first if stale and nvcc is present) the shared library."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if build_if_missing and _build.needs_build():
                _build.build()
            if not os.path.exists(_build.LIB):
                raise RuntimeError(f"libpackb200.so not found at {_build.LIB}; run python -m packing_b200.build")
            L = ctypes.CDLL(_build.LIB)
            for name, args in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = RESTYPES.get(name, ctypes.c_int)
            _lib = L
    return _lib


class PackError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc != 0:
        msg = load().pk_last_error().decode(errors="replace")
        if rc == -1:
            raise ValueError(f"{what}: {msg}")
        if rc == -4:
            raise ValueError(f"{what}: {msg}")
        raise PackError(f"{what} failed ({rc}): {msg}")


def default_geometry(tree_expansion: float = 20 * (1.000001 - 1)) -> PkGeometry:
    g = PkGeometry()
    check(load().pk_default_geometry(tree_expansion, ctypes.byref(g)), "pk_default_geometry")
    return g


def _dev_index(device) -> int:
    if device is None:
        return torch.cuda.current_device()
    if isinstance(device, int):
        return device
    d = torch.device(device)
    return d.index if d.index is not None else torch.cuda.current_device()


def ensure_init(device: torch.device | int | None = None, geometry: PkGeometry | None = None):
    """pk_init on the given (or current) CUDA device, once per device."""
    if not torch.cuda.is_available():
        raise PackError("packing_b200 needs a CUDA device; no CPU fallback exists")
    dev = _dev_index(device)
    if dev in _inited_devices and geometry is None:
        return
    L = load()
    with torch.cuda.device(dev):
        check(L.pk_init(ctypes.byref(geometry) if geometry is not None else None), "pk_init")
    _inited_devices.add(dev)


def as_tensor(a, name: str) -> torch.Tensor:
    """torch.Tensor view of a CUDA array (torch tensor or any __dlpack__ /
    __cuda_array_interface__ object such as a cupy array), zero copy."""
    if isinstance(a, torch.Tensor):
        return a
    if hasattr(a, "__dlpack__"):
        return torch.from_dlpack(a)
    if hasattr(a, "__cuda_array_interface__"):
        return torch.as_tensor(a, device="cuda")
    raise TypeError(f"{name}: expected a CUDA tensor or a DLPack array, got {type(a).__name__}")


def check_f32(t: torch.Tensor, name: str, shape: tuple | None = None):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA array")
    if t.dtype != torch.float32:
        raise ValueError(f"{name} must have dtype float32, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be C-contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")


def stream_handle(stream=None, device=None) -> int:
    """cudaStream_t as int for a torch stream, a cupy-style stream (.ptr),
    an int, or None (torch's current stream)."""
    if stream is None:
        return torch.cuda.current_stream(device).cuda_stream
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    if hasattr(stream, "ptr"):
        return int(stream.ptr)
    raise TypeError(f"unsupported stream object {type(stream).__name__}")


def ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())
