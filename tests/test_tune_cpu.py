"""Host logic of the launch-shape autotuner (no GPU needed)."""
import json

import pytest

from packing_b200 import tune


def test_feasible_threads_respect_near_list_capacity():
    assert tune.feasible_threads(20) == list(tune.CANDIDATE_THREADS)
    assert tune.feasible_threads(1024) == [128, 160, 192, 224, 256]   # 8 t >= 1023
    for n in (1, 200, 513, 1024):
        assert all(8 * t >= n - 1 for t in tune.feasible_threads(n))


def test_buckets():
    assert tune.bucket(1) == 8 and tune.bucket(8) == 8 and tune.bucket(9) == 16
    assert tune.bucket(200) == 200 and tune.bucket(201) == 256 and tune.bucket(1024) == 1024
    with pytest.raises(ValueError):
        tune.bucket(1025)


def test_sample_batch_shape_and_density():
    x, h = tune.sample_batch(3, 50, seed=1)
    assert x.shape == (3, 50, 3) and h.shape == (3, 3)
    s = 1.3 * (50 * tune.TREE_AREA) ** 0.5
    assert abs(x[..., :2]).max() <= s / 2 and (x[..., 2] >= 0).all()


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "t.json"
    tn = tune.RelaxTuner(0, cache_path=str(path))
    monkeypatch.setattr(tn, "gpu_name", lambda: "TESTGPU")
    monkeypatch.setattr(tn, "measure", lambda nb, spec, hist: {(64, False): 2.0, (128, True): 1.0})
    from packing_b200.cost import CostSpec
    assert tn.best(100, CostSpec(), 10) == (128, True)
    data = json.loads(path.read_text())
    assert data["TESTGPU|n128|area|s1|m10"]["threads"] == 128
    tn2 = tune.RelaxTuner(0, cache_path=str(path))
    monkeypatch.setattr(tn2, "gpu_name", lambda: "TESTGPU")
    monkeypatch.setattr(tn2, "measure", lambda *a: pytest.fail("re-measured"))
    assert tn2.best(97, CostSpec(), 10) == (128, True)
