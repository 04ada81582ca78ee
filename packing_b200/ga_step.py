"""One GA generation step on the GPU, built from the hot-path kernels.

The reference's GA (``core/pack_ga3.py``) is outside this package; this module
composes the three hot-path pieces the way a generation uses them:

1. partner matching: for every (parent, partner) pair, a batched Hungarian
   assignment of the parent's trees to the partner's trees on n x n float32
   costs ``|dc|^2 + |wrap(dtheta)|`` (squared centre distance plus angle
   difference) -- ``lap_batch.solve_lap_batch``;
2. crossover + mutation: the child takes the parent's trees, replaces a
   seeded half of them by their matched partner trees, then gets Gaussian
   pose jitter (position sigma, angle sigma);
3. relaxation of all children in one launch -- ``relax.relax``.
"""
from __future__ import annotations

import math

import torch

from . import lap_batch
from .cost import CostSpec
from .relax import RelaxParams, relax


def matching_costs(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """(B, n, n) float32: |c_a_i - c_b_j|^2 + |wrap(theta_a_i - theta_b_j)|."""
    d = a[:, :, None, :2] - b[:, None, :, :2]
    dt = torch.remainder(a[:, :, None, 2] - b[:, None, :, 2] + math.pi, 2 * math.pi) - math.pi
    return ((d * d).sum(-1) + dt.abs()).to(torch.float32).contiguous()


def generation_step(pop: torch.Tensor, partners: torch.Tensor, h: torch.Tensor, generator: torch.Generator,
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
