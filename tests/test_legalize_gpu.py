"""Snap and the batched legalisation (pack_io.py:28-112 with
kaggle_support.py:824-879): snap against a numpy restatement; legalised
packings are overlap-free in FP64 by both the GPU validator and the
oracle's independent clipping check, with the same bounding side."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.workloads import poses

pytestmark = pytest.mark.gpu


def _snap_np(xyt, h0):
    _, _, txy, _, _, _ = O.geometry()
    x, y, t = xyt[..., 0:1], xyt[..., 1:2], xyt[..., 2:3]
    c, s = np.cos(t), np.sin(t)
    vx = (c * txy[:, 0] - s * txy[:, 1] + x).reshape(len(xyt), -1)
    vy = (s * txy[:, 0] + c * txy[:, 1] + y).reshape(len(xyt), -1)
    x0, x1, y0, y1 = vx.min(1), vx.max(1), vy.min(1), vy.max(1)
    xc, yc = (x0 + x1) / 2, (y0 + y1) / 2
    size = np.maximum(x1 - x0, y1 - y0)
    out = xyt.copy()
    out[..., 0] -= xc[:, None]
    out[..., 1] -= yc[:, None]
    return out, np.minimum(size, h0)


def test_snap_matches_restatement(cuda):
    from packing_b200.legalize import snap
    x = poses(9, 30, seed=4) + np.float32(0.7)
    h = np.tile(np.array([[100.0, 0.3, -0.2]], np.float32), (9, 1))
    h[3, 0] = 1.0                                  # smaller than the box: kept
    xo, ho = snap(torch.from_numpy(x).to(cuda), torch.from_numpy(h).to(cuda))
    rx, rh = _snap_np(x.astype(np.float64), h[:, 0].astype(np.float64))
    np.testing.assert_allclose(xo.cpu().numpy(), rx, rtol=0, atol=2e-5)
    np.testing.assert_allclose(ho[:, 0].cpu().numpy(), rh, rtol=1e-5)
    assert float(ho[:, 1:].abs().sum()) == 0.0


def test_legalize_gives_fp64_legal_packings(cuda):
    from packing_b200.cost import CostSpec
    from packing_b200.legalize import legalize
    from packing_b200.relax import RelaxParams, relax
    E, n = 12, 20
    x = torch.from_numpy(poses(E, n, seed=8)).to(cuda)
    h = torch.zeros((E, 3), device=cuda)
    h[:, 0] = 1.3 * np.sqrt(n * 0.2456875) + 1.5
    # start from relaxed but still overlapping packings (legalisation is the
    # last step of a search, pack_ga3.py:576-581)
    xr, hr, loss, _ = relax(x, h, CostSpec(pair="area", w_area=1e-2, fixed_h=True),
                            RelaxParams(n_iterations=400, history_size=10, max_step=0.01))
    before, _ = O.validate(xr.cpu().numpy().astype(np.float64))
    assert (before > 0).any()
    r = legalize(xr, hr, first_iterations=3000, move_factor=5.0)
    assert bool(r.legal.all())
    ov, side = O.validate(r.xyt.cpu().numpy().astype(np.float64))
    assert (ov == 0).all()
    np.testing.assert_allclose(r.side.cpu().numpy(), side, rtol=1e-12)
    assert bool((r.overlap_cost < 1e-10).all()) or bool(r.legal.all())
    assert int(r.rounds.min()) >= 1
