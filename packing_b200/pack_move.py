"""Drop-in for ``core/pack_move.py``: the GA's offspring moves on the GPU.

The move classes keep the reference's names, fields and defaults
(``pack_move.py:22-1033``): ``MoveRandomTree``, ``JiggleRandomTree``,
``JiggleCluster``, ``Translate``, ``Twist``, ``Crossover``, ``Crossover2`` and
``MoveSelector``.  ``do_move_vec(population, inds_to_do, mate_sol, inds_mate,
generator)`` mutates the rows ``inds_to_do`` of ``population.genotype.xyt``
in place, taking mate trees from ``mate_sol.xyt[inds_mate]``, as the
reference does.  A ``MoveSelector`` (or a single move) is applied in one
launch of ``pk_moves``: one CTA per row chooses the move and applies it.

The population / mate collections are any objects with the fields the
moves read: ``xyt`` (E, n, 3) and ``h`` (E, 3) float32 CUDA tensors and the
class fields of ``Genotype`` below (``kind`` 'square' | 'sym90' | 'sym180',
``edge_spacer``, ``filter_move_locations_with_edge_spacer``,
``filter_move_locations_margin``).  A population may also be given as an
object whose ``genotype`` attribute is such a collection, like the
reference's ``Population``.

Random draws come from the library's Philox4x32-10 stream (``MoveGenerator``:
a seed and a call counter), not from a cupy generator; given the draws, every
move follows the reference's arithmetic.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib

PK_MOVE_RANDOM_TREE, PK_MOVE_JIGGLE_TREE, PK_MOVE_JIGGLE_CLUSTER = 0, 1, 2
PK_MOVE_TRANSLATE, PK_MOVE_TWIST, PK_MOVE_CROSSOVER, PK_MOVE_CROSSOVER2 = 3, 4, 5, 6
GENO_KINDS = {"square": 0, "sym90": 1, "sym180": 2}
DISTANCE_FUNCTIONS = {"stripe": 0, "square": 1, "square90": 2, "square180": 3}
PHENOTYPE_MULT = {"square": 1, "sym90": 4, "sym180": 2}


@dataclass
class EdgeSpacerDummy:
    """Accepts every location (kaggle_support.py:480-486)."""


@dataclass
class EdgeSpacerBasic:
    """Valid: far enough from both edge pairs, or near a corner (kaggle_support.py:489-513)."""
    dist_x: float = 0.5
    dist_y: float = 0.5
    dist_corner: float = 0.0


@dataclass
class Genotype:
    """The fields of a ``SolutionCollection`` the moves read."""
    xyt: torch.Tensor = None
    h: torch.Tensor = None
    kind: str = "square"
    edge_spacer: object = field(default_factory=EdgeSpacerDummy)
    filter_move_locations_with_edge_spacer: bool = False
    filter_move_locations_margin: float = 0.25

    @property
    def N_trees(self) -> int:
        return int(self.xyt.shape[1]) * PHENOTYPE_MULT[self.kind]


class MoveGenerator:
    """Seed and call counter of the moves' Philox stream; every
    ``do_move_vec`` call advances the counter, so successive calls draw
    fresh numbers and a run is reproducible from its seed."""

    def __init__(self, seed: int = 0):
        self.seed = int(seed) & ((1 << 64) - 1)
        self.call = 0

    def take(self) -> tuple[int, int]:
        c = self.call
        self.call += 1
        return self.seed, c


@dataclass
class Move:
    respect_edge_spacer_filter: bool = True

    def _fill(self, m: _lib.PkMove):
        raise NotImplementedError

    def to_c(self) -> _lib.PkMove:
        m = _lib.PkMove()
        m.respect_edge_spacer_filter = int(bool(self.respect_edge_spacer_filter))
        self._fill(m)
        return m

    def do_move_vec(self, population, inds_to_do, mate_sol, inds_mate, generator):
        """Apply the move to rows ``inds_to_do`` of the population (pack_move.py:31-55)."""
        return apply_moves([(self, 1.0)], population, inds_to_do, mate_sol, inds_mate, generator)


@dataclass
class MoveRandomTree(Move):
    """A random tree to a random location and angle (pack_move.py:161-188)."""

    def _fill(self, m):
        m.type = PK_MOVE_RANDOM_TREE


@dataclass
class JiggleRandomTree(Move):
    """A random tree shifted by uniform offsets (pack_move.py:191-224)."""
    max_xy_move: float = 0.1
    max_theta_move: float = np.pi

    def _fill(self, m):
        m.type = PK_MOVE_JIGGLE_TREE
        m.max_xy_move, m.max_theta_move = float(self.max_xy_move), float(self.max_theta_move)


@dataclass
class JiggleCluster(Move):
    """The trees nearest a random centre shifted by uniform offsets (pack_move.py:227-298)."""
    max_xy_move: float = 0.1
    max_theta_move: float = np.pi
    min_N_trees: int = 2
    max_N_trees: int = 8

    def _fill(self, m):
        m.type = PK_MOVE_JIGGLE_CLUSTER
        m.max_xy_move, m.max_theta_move = float(self.max_xy_move), float(self.max_theta_move)
        m.min_n_trees, m.max_n_trees = int(self.min_N_trees), int(self.max_N_trees)


@dataclass
class Translate(Move):
    """All trees shifted by a random offset, wrapped into the square (pack_move.py:301-333)."""

    def _fill(self, m):
        m.type = PK_MOVE_TRANSLATE


@dataclass
class Twist(Move):
    """Trees rotated about a random centre by an angle falling to zero at a
    random radius (pack_move.py:336-382)."""
    min_radius: float = 0.5
    max_radius: float = 2.0

    def _fill(self, m):
        m.type = PK_MOVE_TWIST
        m.min_radius, m.max_radius = float(self.min_radius), float(self.max_radius)


@dataclass
class Crossover(Move):
    """The trees nearest a point replaced by the mate's trees nearest another,
    mirrored / turned by a multiple of 90 degrees about their centre of mass
    (pack_move.py:406-632)."""
    min_N_trees: int = 2
    max_N_trees_ratio: float = 0.5
    simple_mate_location: bool = True

    def _fill(self, m):
        m.type = PK_MOVE_CROSSOVER
        m.min_n_trees = int(self.min_N_trees)
        m.max_n_trees_ratio = float(self.max_N_trees_ratio)
        m.simple_mate_location = int(bool(self.simple_mate_location))


@dataclass
class Crossover2(Move):
    """The trees nearest a stripe or square replaced by the mate's, after
    turning the whole mate (pack_move.py:635-1033)."""
    min_N_trees: int = 2
    max_N_trees_ratio: float = 0.5
    distance_function: str = "stripe"
    decouple_mate_location: bool = False
    use_edge_clearance_when_decoupled: bool = True
    do_90_rotation: bool = True

    def _fill(self, m):
        m.type = PK_MOVE_CROSSOVER2
        m.min_n_trees = int(self.min_N_trees)
        m.max_n_trees_ratio = float(self.max_N_trees_ratio)
        if self.distance_function not in DISTANCE_FUNCTIONS:
            raise ValueError(f"Unknown distance function: {self.distance_function}")
        m.distance_function = DISTANCE_FUNCTIONS[self.distance_function]
        m.decouple_mate_location = int(bool(self.decouple_mate_location))
        m.use_edge_clearance_when_decoupled = int(bool(self.use_edge_clearance_when_decoupled))
        m.do_90_rotation = int(bool(self.do_90_rotation))


@dataclass
class MoveSelector(Move):
    """Each row draws one of ``moves`` (entries ``[Move, name, weight]``) with
    probability proportional to its weight (pack_move.py:119-158)."""
    moves: list = field(default_factory=list)

    def do_move_vec(self, population, inds_to_do, mate_sol, inds_mate, generator):
        entries = [(m[0], float(m[2])) for m in self.moves]
        for mv, _ in entries:
            if isinstance(mv, MoveSelector):
                raise ValueError("a MoveSelector inside a MoveSelector is not supported")
        return apply_moves(entries, population, inds_to_do, mate_sol, inds_mate, generator)


def _collection(obj):
    return obj.genotype if hasattr(obj, "genotype") else obj


def _geno_c(pop, mate) -> _lib.PkGenotype:
    g = _lib.PkGenotype()
    kind = getattr(pop, "kind", "square")
    mkind = getattr(mate, "kind", "square") if mate is not None else kind
    if kind not in GENO_KINDS or mkind not in GENO_KINDS:
        raise ValueError("kind must be 'square', 'sym90' or 'sym180'")
    g.kind, g.mate_kind = GENO_KINDS[kind], GENO_KINDS[mkind]
    g.filter = int(bool(getattr(pop, "filter_move_locations_with_edge_spacer", False)))
    g.margin = float(getattr(pop, "filter_move_locations_margin", 0.25))
    sp = getattr(pop, "edge_spacer", None)
    if sp is None or isinstance(sp, EdgeSpacerDummy):
        g.spacer = 0
    elif isinstance(sp, EdgeSpacerBasic) or all(hasattr(sp, a) for a in ("dist_x", "dist_y", "dist_corner")):
        g.spacer = 1
        g.dist_x, g.dist_y, g.dist_corner = float(sp.dist_x), float(sp.dist_y), float(sp.dist_corner)
    else:
        raise ValueError(f"unsupported edge spacer {type(sp).__name__}")
    return g


def move_set(entries, pop, mate=None) -> _lib.PkMoveSet:
    """The ``PkMoveSet`` of [(move, weight), ...] for a population class."""
    if not 1 <= len(entries) <= _lib.PK_MAX_MOVE_TYPES:
        raise ValueError(f"between 1 and {_lib.PK_MAX_MOVE_TYPES} moves")
    s = _lib.PkMoveSet()
    s.n_moves = len(entries)
    w = np.array([e[1] for e in entries], dtype=np.float64)
    if np.any(w < 0) or w.sum() <= 0:
        raise ValueError("move weights must be non-negative with a positive sum")
    prob = (w / w.sum()).astype(np.float32)        # the reference keeps them in float32
    cum = np.cumsum(prob, dtype=np.float32)
    for i, (mv, _) in enumerate(entries):
        s.moves[i] = mv.to_c()
        s.cum_prob[i] = float(cum[i])
    s.geno = _geno_c(pop, mate)
    return s


def apply_moves(entries, population, inds_to_do, mate_sol, inds_mate, generator, stream=None, check=True):
    """One ``pk_moves`` launch: rows ``inds_to_do`` of the population mutated
    in place.  Returns the chosen entry per row (int32, -1 for none)."""
    pop = _collection(population)
    mate = _collection(mate_sol) if mate_sol is not None else None
    x, h = pop.xyt, pop.h
    _lib.check_f32(x, "population xyt")
    _lib.check_f32(h, "population h", (x.shape[0], 3))
    if not x.is_contiguous() or not h.is_contiguous():
        raise ValueError("population xyt and h must be contiguous")
    dev = x.device
    E, n = int(x.shape[0]), int(x.shape[1])
    idx = torch.as_tensor(inds_to_do, device=dev).to(torch.int32).contiguous()
    C = int(idx.numel())
    s = move_set(entries, pop, mate)
    needs_mate = any(isinstance(e[0], (Crossover, Crossover2)) for e in entries)
    mx = mh = midx = None
    M = 0
    if mate is not None:
        mx, mh = mate.xyt, mate.h
        _lib.check_f32(mx, "mate xyt")
        if tuple(mx.shape[1:]) != (n, 3):
            raise ValueError("mate xyt must be (M, n, 3) with the population's n")
        _lib.check_f32(mh, "mate h", (mx.shape[0], 3))
        if mx.data_ptr() == x.data_ptr():
            raise ValueError("mate_sol must not share the population's xyt")
        M = int(mx.shape[0])
        midx = torch.as_tensor(inds_mate, device=dev).to(torch.int32).contiguous()
        if midx.numel() != C:
            raise ValueError("inds_mate must have one entry per row of inds_to_do")
    elif needs_mate:
        raise ValueError("crossover moves need mate_sol and inds_mate")
    chosen = torch.empty(C, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    if C == 0:
        return chosen
    if isinstance(generator, MoveGenerator):
        seed, call = generator.take()
    else:
        seed, call = int(generator), 0
    _lib.ensure_init(dev)
    with torch.cuda.device(dev):
        rc = _lib.load().pk_moves(_lib.ptr(x), _lib.ptr(h), E, n, _lib.ptr(idx), C, _lib.ptr(mx), _lib.ptr(mh), M,
                                  _lib.ptr(midx), ctypes.byref(s), seed, call, _lib.ptr(chosen), _lib.ptr(status),
                                  ctypes.c_void_p(_lib.stream_handle(stream, dev)))
    _lib.check(rc, "pk_moves")
    if check:
        st = int(status.item())
        if st & 4:
            raise IndexError("inds_to_do or inds_mate out of range (those rows were left unchanged)")
        if st & 2:
            raise ValueError("a move centre request the reference rejects (symmetric genotype with the edge-spacer "
                             "filter, or edge clearance above a quarter of the side)")
        if st & 1:
            raise RuntimeError("a rejection sampler for move centres found no valid location")
    return chosen


def move_draws(seed: int, call: int, row: int, first: int, count: int, device=None) -> torch.Tensor:
    """Draws first .. first+count-1 of row position ``row`` (float64, device)."""
    dev = torch.device("cuda", _lib._dev_index(device))
    _lib.ensure_init(dev)
    out = torch.empty(max(count, 1), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        rc = _lib.load().pk_move_draws(int(seed), int(call), int(row), int(first), int(count), _lib.ptr(out),
                                       ctypes.c_void_p(_lib.stream_handle(None, dev)))
    _lib.check(rc, "pk_move_draws")
    return out[:count]
