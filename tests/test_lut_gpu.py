"""LUT path: the GPU-built table against the FP64 oracle area, and the LUT
cost kernel against the oracle restatement of pack_cuda_lut."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.workloads import poses

pytestmark = pytest.mark.gpu


def _small_lut(cuda, quad=False):
    from packing_b200.pack_cuda_lut import LookupTable
    return LookupTable.build_from_kernel("area", N_x=64, N_y=64, N_theta=48, trim_zeros=True,
                                         apply_quadratic_transform=quad, device=cuda)


def test_lut_values_match_oracle_area(cuda):
    lut = _small_lut(cuda)
    vals = lut.lut_d.cpu().numpy()
    rng = np.random.default_rng(0)
    idx = np.stack([rng.integers(0, s, 300) for s in vals.shape], 1)
    xyt = np.zeros((300, 2, 3))
    xyt[:, 1, 0] = lut.X[idx[:, 0]]
    xyt[:, 1, 1] = lut.Y[idx[:, 1]]
    xyt[:, 1, 2] = lut.theta[idx[:, 2]]
    oc, _ = O.pair_cost(xyt, False, grad=False)
    np.testing.assert_allclose(vals[idx[:, 0], idx[:, 1], idx[:, 2]], oc, rtol=1e-5, atol=2e-6)


@pytest.mark.parametrize("quad", [False, True])
def test_lut_cost_matches_oracle(cuda, quad):
    from packing_b200 import pack_cuda_lut
    lut = _small_lut(cuda, quad)
    x = poses(16, 60, seed=3)
    xt = torch.from_numpy(x).to(cuda)
    c = torch.empty(16, device=cuda)
    g = torch.empty_like(xt)
    pack_cuda_lut.overlap_multi_ensemble(xt, c, lut, g)
    b = (lut.X_min, lut.X_max, lut.Y_min, lut.Y_max, lut.theta_min, lut.theta_max)
    oc, og = O.lut_cost(list(x.astype(np.float64)), lut.lut_d.cpu().numpy(), b, quad, O.geometry()[3])
    np.testing.assert_allclose(c.cpu().numpy(), oc, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(g.cpu().numpy(), np.stack(og), rtol=1e-3, atol=1e-3)


def test_lut_approximates_analytic_area(cuda):
    """With a fine table the LUT cost tracks the exact overlap area."""
    from packing_b200 import pack_cuda, pack_cuda_lut
    from packing_b200.pack_cuda_lut import LookupTable
    lut = LookupTable.build_from_kernel("area", N_x=256, N_y=256, N_theta=360, trim_zeros=False, device=cuda)
    x = torch.from_numpy(poses(32, 100, seed=5)).to(cuda)
    c1 = torch.empty(32, device=cuda)
    c2 = torch.empty(32, device=cuda)
    pack_cuda_lut.overlap_multi_ensemble(x, c1, lut)
    pack_cuda.overlap_multi_ensemble(x, x, False, out_cost=c2)
    np.testing.assert_allclose(c1.cpu().numpy(), c2.cpu().numpy(), rtol=2e-2)


def test_lut_ragged_equals_uniform(cuda):
    from packing_b200 import pack_cuda_lut
    lut = _small_lut(cuda)
    sizes = [5, 200, 17, 64, 1]
    xs = [poses(1, s, seed=s)[0] for s in sizes]
    flat = torch.from_numpy(np.concatenate(xs)).to(cuda)
    off = torch.tensor(np.concatenate([[0], np.cumsum(sizes)]), dtype=torch.int32, device=cuda)
    c = torch.empty(len(sizes), device=cuda)
    g = torch.empty_like(flat)
    pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, c, lut, g)
    o = np.concatenate([[0], np.cumsum(sizes)])
    for e, s in enumerate(sizes):
        xt = torch.from_numpy(xs[e][None]).to(cuda)
        cu = torch.empty(1, device=cuda)
        gu = torch.empty_like(xt)
        pack_cuda_lut.overlap_multi_ensemble(xt, cu, lut, gu)
        assert float(cu[0]) == float(c[e])
        assert torch.equal(gu[0], g[o[e]:o[e + 1]])


def test_ragged_size_classes_equal_one_launch(cuda):
    """The ragged LUT cost and the ragged compound cost, launched per size
    class side by side, give the bits of one launch."""
    from packing_b200 import pack_cuda_lut
    from packing_b200.classes import ragged_plan
    from packing_b200.cost import CostSpec, compound_cost
    lut = _small_lut(cuda, quad=True)
    rng = np.random.default_rng(11)
    sizes = [int(s) for s in np.round(np.exp(rng.uniform(np.log(2), np.log(260), size=300)))]
    xs = [poses(1, s, seed=700 + k)[0] for k, s in enumerate(sizes)]
    flat = torch.from_numpy(np.concatenate(xs)).to(cuda)
    off = torch.tensor(np.concatenate([[0], np.cumsum(sizes)]), dtype=torch.int32, device=cuda)
    order, classes = ragged_plan(sizes, cuda)
    assert len(classes) >= 5
    E = len(sizes)
    c1, c2 = torch.empty(E, device=cuda), torch.empty(E, device=cuda)
    g1, g2 = torch.empty_like(flat), torch.empty_like(flat)
    pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, c1, lut, g1, n_max=max(sizes))
    pack_cuda_lut.overlap_multi_ensemble_ragged(flat, off, c2, lut, g2, n_max=max(sizes), order=order,
                                                classes=classes)
    assert torch.equal(c1, c2) and torch.equal(g1, g2)
    h = torch.from_numpy(np.concatenate([np.array([[np.sqrt(s * 0.2456875) * 1.3, 0, 0]], np.float32)
                                         for s in sizes])).to(cuda)
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=1e-2, fixed_h=False)
    a = compound_cost(flat, h, spec, offsets=off, n_max=max(sizes))
    b = compound_cost(flat, h, spec, offsets=off, n_max=max(sizes), order=order, classes=classes)
    for u, v in zip(a, b):
        assert torch.equal(u, v)
