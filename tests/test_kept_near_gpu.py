"""Kept near lists in the fused relaxation.

The fused relaxation builds its near-pair list with a skin and reuses it, with
no cell grid, while no tree has moved far enough to matter.  The one-shot cost
kernel behind the drop-in ``lbfgs`` never keeps a list.  The two follow the
same iterates bit for bit only if every reused list yields exactly the pairs
that a fresh grid would: these tests compare them on layouts that reach each
branch.
- A list that overflows the near list falls back to the chunked grid path.
- Large coordinates stress the displacement bound's rounding.
- Symmetric images, the LUT pair term and a step bound too large for kept
  lists are covered too.
"""
import numpy as np
import pytest
import torch

from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu


def _layout(kind, E, seed):
    rng = np.random.default_rng(seed)
    if kind == "headline":
        n = 200
        return poses(E, n, seed=seed), square_h(E, n)
    if kind == "dense":
        # 300 trees in a 6 x 6 square: about 7 000 pairs lie within the kept
        # list's distance, far more than its 2 048 entries at 256 threads, so
        # every evaluation falls back to the chunked grid path
        n = 300
        xy = rng.uniform(-3.0, 3.0, size=(E, n, 2))
    elif kind == "spread":
        # clusters of four overlapping trees about 1 000 units apart
        n = 64
        c = rng.uniform(-1000.0, 1000.0, size=(E, n // 4, 1, 2))
        xy = (c + rng.uniform(-0.4, 0.4, size=(E, n // 4, 4, 2))).reshape(E, n, 2)
    else:
        raise ValueError(kind)
    th = rng.uniform(0.0, 2 * np.pi, size=(E, n, 1))
    xyt = np.concatenate([xy, th], axis=2).astype(np.float32)
    h = np.zeros((E, 3), dtype=np.float32)
    h[:, 0] = 2.0 * float(np.abs(xy).max()) + 2.0
    return xyt, h


def _dropin_and_fused(cuda, xyt, h, spec, iters, max_step, hist=10):
    from packing_b200.cost import compound_cost
    from packing_b200.lbfgs_torch_parallel import lbfgs
    from packing_b200.relax import RelaxParams, relax
    E, n, _ = xyt.shape
    ng = n // spec.symmetry if spec.symmetry > 1 else n

    def f(x, is_main):
        c, g, gh = compound_cost(x[:, :3 * ng].reshape(E, ng, 3).contiguous(), x[:, 3 * ng:].contiguous(), spec)
        return c, torch.cat([g.reshape(E, -1), gh], 1)

    x0 = xyt[:, :ng]
    x = torch.from_numpy(np.concatenate([x0.reshape(E, -1), h], 1)).to(cuda)
    lbfgs(f, x, max_iter=iters, history_size=hist, max_step=max_step, tolerance_grad=0, tolerance_change=0)
    counters = torch.zeros(6, dtype=torch.int64, device=cuda)
    prm = RelaxParams(n_iterations=iters, history_size=hist, max_step=max_step, final_eval=True, counters=counters)
    xr, hr, loss, it = relax(torch.from_numpy(np.ascontiguousarray(x0)).to(cuda), torch.from_numpy(h).to(cuda),
                             spec, prm)
    return x[:, :3 * ng].reshape(E, ng, 3), xr, it, counters.cpu().numpy()


def _area_spec(symmetry=1):
    from packing_b200.cost import CostSpec
    return CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True, symmetry=symmetry)


@pytest.mark.parametrize("kind,iters", [("headline", 60), ("dense", 25), ("spread", 40)])
def test_kept_lists_match_the_one_shot_kernel(cuda, kind, iters):
    xyt, h = _layout(kind, 4, seed=3)
    xd, xr, it, _ = _dropin_and_fused(cuda, xyt, h, _area_spec(), iters, 0.01)
    assert torch.all(it == iters)
    assert torch.equal(xr, xd)


def test_kept_lists_are_reused(cuda):
    """At max_step 0.01 a list serves several evaluations: the centre tests
    per evaluation fall well below those of a grid built every time (the
    step bound 0.05 keeps no lists)."""
    xyt, h = _layout("headline", 4, seed=5)
    per_eval = []
    for max_step in (0.01, 0.05):
        _, _, _, cnt = _dropin_and_fused(cuda, xyt, h, _area_spec(), 40, max_step)
        per_eval.append(cnt[0] / cnt[3])
    assert per_eval[0] < 0.8 * per_eval[1]


def test_kept_lists_off_for_large_steps(cuda):
    xyt, h = _layout("headline", 2, seed=6)
    xd, xr, it, _ = _dropin_and_fused(cuda, xyt, h, _area_spec(), 30, 0.05)
    assert torch.equal(xr, xd)


def test_kept_lists_with_symmetric_images(cuda):
    """A 180-degree symmetric packing: the images' displacements bound the
    list's validity like the genotype trees'."""
    n = 100
    xyt = poses(3, 2 * n, seed=8)
    h = square_h(3, 2 * n)
    xd, xr, it, _ = _dropin_and_fused(cuda, xyt, h, _area_spec(symmetry=2), 40, 0.01)
    assert torch.equal(xr, xd)


def test_kept_lists_with_the_lut_pair_term(cuda):
    from packing_b200.cost import CostSpec
    from packing_b200.pack_cuda_lut import LookupTable
    lut = LookupTable.build_from_kernel("area", N_x=64, N_y=64, N_theta=48, trim_zeros=True, device=cuda)
    spec = CostSpec(pair="lut", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=True, lut=lut)
    xyt, h = _layout("headline", 3, seed=9)
    xd, xr, it, _ = _dropin_and_fused(cuda, xyt, h, spec, 40, 0.01)
    assert torch.equal(xr, xd)
