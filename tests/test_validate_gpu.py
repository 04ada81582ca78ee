"""FP64 legality and bounding side against the oracle (pack_metric.py
semantics: interiors may not intersect, touching is legal)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.workloads import poses, square_h

pytestmark = pytest.mark.gpu


def _val(x, dev, dtype=torch.float64):
    from packing_b200.validate import validate
    ov, side = validate(torch.from_numpy(np.asarray(x)).to(dev, dtype))
    return ov.cpu().numpy(), side.cpu().numpy()


def test_random_packings_match_oracle(cuda):
    x = poses(16, 60, seed=3).astype(np.float64)
    ov, side = _val(x, cuda)
    oov, oside = O.validate(x)
    assert np.array_equal(ov, oov)
    np.testing.assert_allclose(side, oside, rtol=1e-12)


def test_float32_input(cuda):
    x = poses(4, 30, seed=4)
    ov, side = _val(x, cuda, torch.float32)
    oov, oside = O.validate(x.astype(np.float64))
    assert np.array_equal(ov, oov)
    np.testing.assert_allclose(side, oside, rtol=1e-12)


def test_gap_touch_overlap(cuda):
    # two upright trees side by side; the widest tier is 0.7 wide
    x = np.array([[[0, 0, 0], [0.7 + 1e-7, 0, 0]],
                  [[0, 0, 0], [0.7, 0, 0]],
                  [[0, 0, 0], [0.6, 0, 0]],
                  [[0, 0, 0], [0, 0, np.pi]],
                  [[0, 0, 0], [0, 1.0 + 1e-7, 0]],
                  [[0, 0, 0], [0.3, 0.3, 0.5]]])
    ov, side = _val(x, cuda)
    oov, oside = O.validate(x)
    assert list(ov) == [0, 0, 1, 1, 0, 1]
    assert np.array_equal(ov, oov)
    np.testing.assert_allclose(side, oside, rtol=1e-14)
    assert side[0] == pytest.approx(1.4 + 1e-7, rel=1e-12)


def test_relaxed_packings_become_legal(cuda):
    """A relaxation of a loose packing ends FP64-legal, and the FP64 side
    agrees with the oracle's to 1e-6 relative (here: to 1e-12)."""
    from packing_b200.cost import CostSpec
    from packing_b200.relax import RelaxParams, relax
    n, E = 20, 32
    x = torch.from_numpy(poses(E, n, seed=8, side_factor=2.0)).to(cuda)
    h = torch.from_numpy(square_h(E, n) * 1.5).to(cuda)
    spec = CostSpec(pair="area", w_pair=1.0, w_boundary=1.0, w_area=0.0, fixed_h=True)
    xr, hr, loss, it = relax(x, h, spec, RelaxParams(n_iterations=300, history_size=10, max_step=0.01))
    ov, side = _val(xr.double().cpu().numpy(), cuda)
    oov, oside = O.validate(xr.double().cpu().numpy())
    assert np.array_equal(ov, oov)
    np.testing.assert_allclose(side, oside, rtol=1e-12)
    assert (ov == 0).mean() > 0.9
