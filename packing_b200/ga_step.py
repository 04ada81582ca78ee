"""One GA offspring generation on the GPU, built from the hot-path kernels.

The reference's GA (``core/pack_ga3.py``) produces a generation's offspring
as ``_generate_offspring`` does (``pack_ga3.py:1343-1431``):

1. clone the chosen parents into the new population;
2. apply the move selector to every clone, with a mate from the old
   population (never the parent itself) -- here ``pk_moves``, one launch for
   the whole selector (``pack_move.MoveSelector``);
3. canonicalise the genotypes (a no-op for plain squares);
4. relax the offspring with the GA's fitness cost (``pack_ga3.py:1475-1477``:
   area 1e-2, boundary, exact-separation LUT) -- one ``relax`` launch.

``default_moves()`` is the reference GA's move selector (``pack_ga3.py:1084-1115``).

``crossover_jitter_step`` is the matched-crossover generation the batched
Hungarian serves: every parent's trees are assigned to its partner's trees
by ``lap_batch.solve_lap_batch`` on n x n costs (``matching_costs``: squared
centre distance plus angle difference), the child takes a seeded half of
the matched partner trees, gets Gaussian pose jitter, and is relaxed.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import lap_batch
from . import pack_move as PM
from .cost import CostSpec
from .relax import RelaxParams, relax


def default_moves() -> PM.MoveSelector:
    """The GA's default move selector (pack_ga3.py:1084-1115)."""
    return PM.MoveSelector(moves=[
        [PM.MoveRandomTree(), "MoveRandomTree", 1.0],
        [PM.JiggleRandomTree(max_xy_move=0.05, max_theta_move=np.pi / 6), "JiggleTreeSmall", 1.0],
        [PM.JiggleRandomTree(max_xy_move=0.1, max_theta_move=np.pi), "JiggleTreeBig", 1.0],
        [PM.JiggleCluster(max_xy_move=0.05, max_theta_move=np.pi / 6), "JiggleClusterSmall", 1.0],
        [PM.JiggleCluster(max_xy_move=0.1, max_theta_move=np.pi), "JiggleClusterBig", 1.0],
        [PM.Translate(), "Translate", 1.0],
        [PM.Twist(), "Twist", 1.0],
        [PM.Crossover(), "Crossover", 2.0],
        [PM.Crossover2(), "Crossover2", 2.0],
    ])


def fitness_spec(lut) -> CostSpec:
    """The GA's fitness cost on an exact-separation table
    (``LookupTable.build_exact_separation``) at fixed h."""
    return CostSpec(pair="lut", lut=lut, w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True)


def matching_costs(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """(B, n, n) float32: |c_a_i - c_b_j|^2 + |wrap(theta_a_i - theta_b_j)|."""
    d = a[:, :, None, :2] - b[:, None, :, :2]
    dt = torch.remainder(a[:, :, None, 2] - b[:, None, :, 2] + math.pi, 2 * math.pi) - math.pi
    return ((d * d).sum(-1) + dt.abs()).to(torch.float32).contiguous()


def generation_step(pop: torch.Tensor, h: torch.Tensor, parents: torch.Tensor, mates: torch.Tensor,
                    generator: PM.MoveGenerator, spec: CostSpec, moves: PM.MoveSelector | None = None,
                    iterations: int = 80, history: int = 3, max_step: float = 0.1):
    """pop (P, n, 3) and h (P, 3) the old population; parents and mates (C,)
    indices into it.  Returns (offspring relaxed (C, n, 3), their h, loss
    (C,), chosen move per offspring (C,)).  The relaxation defaults are the
    rough relaxer's: OptimizerBFGS (history 3, pack_dynamics.py:33-39) with
    80 iterations and max_step 0.1 (pack_ga3.py:1481-1486)."""
    moves = moves or default_moves()
    parents = parents.to(pop.device, torch.long)
    child = PM.Genotype(pop.index_select(0, parents).contiguous(), h.index_select(0, parents).contiguous())
    old = PM.Genotype(pop, h)
    C = int(parents.numel())
    chosen = moves.do_move_vec(child, torch.arange(C, device=pop.device), old, mates.to(pop.device), generator)
    out, hout, loss, _ = relax(child.xyt, child.h, spec,
                               RelaxParams(n_iterations=iterations, history_size=history, max_step=max_step,
                                           final_eval=True))
    return out, hout, loss, chosen


def crossover_jitter_step(pop: torch.Tensor, partners: torch.Tensor, h: torch.Tensor, generator: torch.Generator,
                          sigma_xy: float = 0.05, sigma_deg: float = 5.0, iterations: int = 100,
                          spec: CostSpec = CostSpec(), history: int = 10, max_step: float = 0.01):
    """pop (P, n, 3), partners (P,) int64 indices into pop, h (P, 3).
    Returns (children relaxed (P, n, 3), loss (P,), row_match (P, n))."""
    P, n, _ = pop.shape
    mates = pop[partners]
    C = matching_costs(pop, mates)
    row_match, _ = lap_batch.solve_lap_batch(C)
    matched = torch.gather(mates, 1, row_match.long().clamp_min(0)[:, :, None].expand(P, n, 3))
    take = torch.rand((P, n, 1), generator=generator, device=pop.device) < 0.5
    child = torch.where(take, matched, pop)
    noise = torch.randn((P, n, 3), generator=generator, device=pop.device)
    noise[:, :, :2] *= sigma_xy
    noise[:, :, 2] *= math.radians(sigma_deg)
    child = (child + noise).contiguous()
    out, _, loss, _ = relax(child, h, spec, RelaxParams(n_iterations=iterations, history_size=history,
                                                        max_step=max_step, final_eval=True))
    return out, loss, row_match
