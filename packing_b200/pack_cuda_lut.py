"""Drop-in for ``core/pack_cuda_lut.py``: LUT-based tree-pair cost.

``LookupTable`` keeps the reference's fields and grid conventions
(``pack_cuda_lut.py:30-254``): ``vals[ix, iy, it]`` over X (the non-negative
half plus one negative sample; negative x is served by mirror symmetry), Y
and theta; optional ``max(0, v)^2`` per pair.  The device copy is a torch
tensor (``lut_d``).  ``overlap_multi_ensemble`` (``:783``) evaluates the sum
over pairs ``i < j`` within ``2R`` of the trilinear LUT value with its
analytic gradient on both trees; ragged batches are served by
``overlap_multi_ensemble_ragged`` in one launch (the reference needs one
launch per distinct tree count).

``LookupTable.build_from_kernel`` builds the table on the GPU from the
analytic overlap-area (or separation) kernel, the same quantity
``CollisionCost._ensure_lut_initialized`` tabulates
(``pack_cost.py:322-377``); ``build_from_function`` accepts any CPU
``eval_fn`` exactly like the reference.  ``build_exact_separation`` builds
the production table of ``CollisionCostExactSeparation``
(``pack_cost.py:1144-1215``) -- the signed Minkowski separation the
reference tabulates slice by slice with shapely -- on the GPU in FP64.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib


def tree_max_radius() -> float:
    return float(_lib.default_geometry().max_radius)


@dataclass
class LookupTable:
    X: np.ndarray
    Y: np.ndarray
    theta: np.ndarray
    vals: object
    apply_quadratic_transform: bool = False
    lut_d: Optional[torch.Tensor] = field(default=None, repr=False)

    def __post_init__(self):
        shape = tuple(self.vals.shape)
        if len(shape) != 3:
            raise ValueError(f"vals must be 3-D, got shape {shape}")
        n_x, n_y, n_t = shape
        self.X = np.asarray(self.X, dtype=np.float32)
        self.Y = np.asarray(self.Y, dtype=np.float32)
        self.theta = np.asarray(self.theta, dtype=np.float32)
        if len(self.X) != n_x or len(self.Y) != n_y or len(self.theta) != n_t:
            raise ValueError(f"LUT shape mismatch: vals={shape}, X={len(self.X)}, Y={len(self.Y)}, "
                             f"theta={len(self.theta)}")
        self.N_x, self.N_y, self.N_theta = n_x, n_y, n_t
        self.X_min, self.X_max = float(self.X[0]), float(self.X[-1])
        self.Y_min, self.Y_max = float(self.Y[0]), float(self.Y[-1])
        self.theta_min, self.theta_max = float(self.theta[0]), float(self.theta[-1])
        self.grid_dx = (self.X_max - self.X_min) / (n_x - 1) if n_x > 1 else 0.0
        self.grid_dy = (self.Y_max - self.Y_min) / (n_y - 1) if n_y > 1 else 0.0
        self.grid_dtheta = (self.theta_max - self.theta_min) / (n_t - 1) if n_t > 1 else 0.0
        self._prepare_gpu_resources()

    def _prepare_gpu_resources(self, device=None):
        v = self.vals
        if isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float32 and v.is_contiguous():
            self.lut_d = v
        else:
            t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32))
            self.lut_d = t.to(device=device or "cuda", dtype=torch.float32).contiguous()

    def c_struct(self) -> _lib.PkLut:
        L = _lib.PkLut()
        L.vals = self.lut_d.data_ptr()
        L.nx, L.ny, L.nt = self.N_x, self.N_y, self.N_theta
        L.x_min, L.x_max = self.X_min, self.X_max
        L.y_min, L.y_max = self.Y_min, self.Y_max
        L.t_min, L.t_max = self.theta_min, self.theta_max
        L.quadratic = int(bool(self.apply_quadratic_transform))
        return L

    def nbytes(self) -> int:
        return self.N_x * self.N_y * self.N_theta * 4

    @staticmethod
    def default_grid(N_x=400, N_y=400, N_theta=400):
        """The reference's default axes (pack_cuda_lut.py:127-135)."""
        R = tree_max_radius()
        X = np.linspace(-2 * R, 2 * R, N_x, dtype=np.float32)
        X = X[N_x // 2 - 1:]
        assert X[0] < 0
        Y = np.linspace(-2 * R, 2 * R, N_y, dtype=np.float32)
        theta = np.linspace(-np.pi, np.pi, N_theta, dtype=np.float32)
        return X, Y, theta

    @classmethod
    def build_from_function(cls, eval_fn, X=None, Y=None, theta=None, N_x=400, N_y=400, N_theta=400,
                            trim_zeros=True, verbose=True) -> "LookupTable":
        """Tabulate a CPU ``eval_fn(dx, dy, theta) -> costs`` (pack_cuda_lut.py:90-169)."""
        dX, dY, dT = cls.default_grid(N_x, N_y, N_theta)
        X = dX if X is None else np.asarray(X, np.float32)
        Y = dY if Y is None else np.asarray(Y, np.float32)
        theta = dT if theta is None else np.asarray(theta, np.float32)
        vals = np.zeros((len(X), len(Y), len(theta)), dtype=np.float32)
        gx, gy = np.meshgrid(X, Y, indexing="ij")
        for t_idx, t_val in enumerate(theta):
            vals[:, :, t_idx] = np.asarray(eval_fn(gx.ravel(), gy.ravel(), t_val)).reshape(len(X), len(Y))
        if trim_zeros:
            X, Y, theta, vals = cls._trim_zero_edges(X, Y, theta, vals, verbose=verbose)
        return cls(X=X, Y=Y, theta=theta, vals=vals)

    @classmethod
    def build_from_kernel(cls, pair="area", X=None, Y=None, theta=None, N_x=400, N_y=400, N_theta=400,
                          trim_zeros=True, apply_quadratic_transform=False, device=None) -> "LookupTable":
        """Tabulate the analytic pair cost ('area' or 'sep') on the GPU."""
        dX, dY, dT = cls.default_grid(N_x, N_y, N_theta)
        X = dX if X is None else np.asarray(X, np.float32)
        Y = dY if Y is None else np.asarray(Y, np.float32)
        theta = dT if theta is None else np.asarray(theta, np.float32)
        dev = torch.device(device or "cuda")
        _lib.ensure_init(dev)
        Xd = torch.from_numpy(X).to(dev)
        Yd = torch.from_numpy(Y).to(dev)
        Td = torch.from_numpy(theta).to(dev)
        vals = torch.empty((len(X), len(Y), len(theta)), device=dev, dtype=torch.float32)
        mode = {"area": _lib.PK_PAIR_AREA, "sep": _lib.PK_PAIR_SEP}[pair]
        with torch.cuda.device(dev):
            rc = _lib.load().pk_lut_build(_lib.ptr(Xd), len(X), _lib.ptr(Yd), len(Y), _lib.ptr(Td), len(theta), mode,
                                          _lib.ptr(vals), ctypes.c_void_p(_lib.stream_handle(None, dev)))
        _lib.check(rc, "pk_lut_build")
        if trim_zeros:
            X, Y, theta, v = cls._trim_zero_edges(X, Y, theta, vals.cpu().numpy(), verbose=False)
            vals = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
        return cls(X=X, Y=Y, theta=theta, vals=vals, apply_quadratic_transform=apply_quadratic_transform)

    @classmethod
    def build_exact_separation(cls, X=None, Y=None, theta=None, N_x=900, N_y=900, N_theta=900, trim_zeros=True,
                               device=None) -> "LookupTable":
        """The table of ``CollisionCostExactSeparation`` (pack_cost.py:1144-1215):
        the signed Minkowski separation of pack_minkowski.separation_distance
        tabulated on the reference's default 900^3 grid, built on the GPU in
        FP64 and stored as float32, with the per-pair ``max(0, v)^2``
        transform on."""
        dX, dY, dT = cls.default_grid(N_x, N_y, N_theta)
        X = dX if X is None else np.asarray(X, np.float32)
        Y = dY if Y is None else np.asarray(Y, np.float32)
        theta = dT if theta is None else np.asarray(theta, np.float32)
        dev = torch.device(device or "cuda")
        _lib.ensure_init(dev)
        Xd = torch.from_numpy(np.ascontiguousarray(X)).to(dev)
        Yd = torch.from_numpy(np.ascontiguousarray(Y)).to(dev)
        Td = torch.from_numpy(np.ascontiguousarray(theta)).to(dev)
        vals = torch.empty((len(X), len(Y), len(theta)), device=dev, dtype=torch.float32)
        with torch.cuda.device(dev):
            rc = _lib.load().pk_lut_build_exact_sep(_lib.ptr(Xd), len(X), _lib.ptr(Yd), len(Y), _lib.ptr(Td),
                                                    len(theta), _lib.ptr(vals),
                                                    ctypes.c_void_p(_lib.stream_handle(None, dev)))
        _lib.check(rc, "pk_lut_build_exact_sep")
        if trim_zeros:
            X, Y, theta, vals = cls._trim_zero_edges_device(X, Y, theta, vals)
        return cls(X=X, Y=Y, theta=theta, vals=vals, apply_quadratic_transform=True)

    @staticmethod
    def _trim_ranges(mx_x, mx_y, mx_t):
        """Index ranges kept by the trim: the positive span of each axis's
        maxima, widened by one row/column on X and Y (pack_cuda_lut.py:171-254)."""
        def rng(mx, keep):
            pos = np.where(mx > 0)[0]
            if len(pos) == 0:
                return 0, len(mx) - 1
            if keep:
                return max(0, pos[0] - 1), min(len(mx) - 1, pos[-1] + 1)
            return pos[0], pos[-1]
        return rng(mx_x, True), rng(mx_y, True), rng(mx_t, False)

    @classmethod
    def _trim_zero_edges_device(cls, X, Y, theta, vals):
        """``_trim_zero_edges`` on a device table, without copying it to the host."""
        (xs, xe), (ys, ye), (ts, te) = cls._trim_ranges(vals.amax(dim=(1, 2)).cpu().numpy(),
                                                        vals.amax(dim=(0, 2)).cpu().numpy(),
                                                        vals.amax(dim=(0, 1)).cpu().numpy())
        v = vals[xs:xe + 1, ys:ye + 1, ts:te + 1].contiguous()
        return X[xs:xe + 1], Y[ys:ye + 1], theta[ts:te + 1], v

    @classmethod
    def _trim_zero_edges(cls, X, Y, theta, vals, verbose=True):
        """Drop all-non-positive edge slabs, keeping one non-positive row/column
        at each X and Y edge (pack_cuda_lut.py:171-254)."""
        N_x, N_y, N_t = vals.shape
        (xs, xe), (ys, ye), (ts, te) = cls._trim_ranges(np.max(vals, axis=(1, 2)), np.max(vals, axis=(0, 2)),
                                                        np.max(vals, axis=(0, 1)))
        out = (X[xs:xe + 1], Y[ys:ye + 1], theta[ts:te + 1], vals[xs:xe + 1, ys:ye + 1, ts:te + 1])
        if verbose:
            print(f"Trimming non-positive edges: X {N_x}->{len(out[0])}, Y {N_y}->{len(out[1])}, "
                  f"theta {N_t}->{len(out[2])}")
        return out


def overlap_multi_ensemble(xyt, out_cost, lut: LookupTable, out_grads=None, stream=None):
    """Sum over pairs i < j within 2R of the LUT value at the relative pose
    (in tree i's frame) with optional max(0, v)^2, and its gradient on both
    trees.  Reference ``pack_cuda_lut.py:783-862``."""
    x = _lib.as_tensor(xyt, "xyt")
    if x.ndim != 3 or x.shape[2] != 3:
        raise ValueError(f"xyt shape: {tuple(x.shape)}")
    _lib.check_f32(x, "xyt")
    E, n = int(x.shape[0]), int(x.shape[1])
    c = _lib.as_tensor(out_cost, "out_cost")
    _lib.check_f32(c, "out_cost", (E,))
    g = None
    if out_grads is not None:
        g = _lib.as_tensor(out_grads, "out_grads")
        _lib.check_f32(g, "out_grads", (E, n, 3))
    if E == 0:
        return
    _lib.ensure_init(x.device)
    L = lut.c_struct()
    with torch.cuda.device(x.device):
        rc = _lib.load().pk_overlap_lut(_lib.ptr(x), None, E, n, ctypes.byref(L), _lib.ptr(c), _lib.ptr(g),
                                        ctypes.c_void_p(_lib.stream_handle(stream, x.device)))
    _lib.check(rc, "pack_cuda_lut.overlap_multi_ensemble")


def overlap_multi_ensemble_ragged(xyt_packed, offsets, out_cost, lut: LookupTable, out_grads=None, n_max=None,
                                  stream=None, order=None, classes=None):
    """Ragged form: ``xyt_packed`` (sum n, 3), int32 device ``offsets``
    (E+1,), ``n_max`` >= every instance size (read from offsets if None).
    With a largest-first ``order`` and its ``classes``
    (``classes.ragged_plan``): one launch per size class, side by side,
    bit-identical to one launch."""
    x = _lib.as_tensor(xyt_packed, "xyt_packed")
    _lib.check_f32(x, "xyt_packed")
    off = _lib.as_tensor(offsets, "offsets")
    if off.dtype != torch.int32 or not off.is_cuda:
        raise ValueError("offsets must be a CUDA int32 vector")
    E = int(off.shape[0]) - 1
    if n_max is None:
        n_max = int((off[1:] - off[:-1]).max().item()) if E > 0 else 0
    c = _lib.as_tensor(out_cost, "out_cost")
    _lib.check_f32(c, "out_cost", (E,))
    g = None
    if out_grads is not None:
        g = _lib.as_tensor(out_grads, "out_grads")
        _lib.check_f32(g, "out_grads", tuple(x.shape))
    if E == 0:
        return
    _lib.ensure_init(x.device)
    L = lut.c_struct()
    if classes is not None:
        from .cost import launch_cost_classes
        cs = _lib.PkCostSpec()
        cs.pair_mode = _lib.PK_PAIR_LUT
        cs.w_pair = 1.0
        cs.lut = L
        launch_cost_classes(x, off, order, E, int(n_max), None, cs, c, g, None, classes, stream,
                            "pack_cuda_lut.overlap_multi_ensemble_ragged")
        return
    with torch.cuda.device(x.device):
        rc = _lib.load().pk_overlap_lut(_lib.ptr(x), _lib.ptr(off), E, int(n_max), ctypes.byref(L), _lib.ptr(c),
                                        _lib.ptr(g), ctypes.c_void_p(_lib.stream_handle(stream, x.device)))
    _lib.check(rc, "pack_cuda_lut.overlap_multi_ensemble_ragged")
