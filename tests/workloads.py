"""Seeded synthetic inputs with the shapes of the benchmark configurations
(synthetic stand-ins: the reference publishes no dataset)."""
import numpy as np

TREE_AREA = 0.2456875


def poses(E, n, seed=0, side_factor=1.3):
    """x, y ~ U(-s/2, s/2), s = side_factor * sqrt(n * tree area);
    theta ~ U(0, 360 deg) in radians.  float32 (E, n, 3)."""
    rng = np.random.default_rng(seed)
    s = side_factor * np.sqrt(n * TREE_AREA)
    xy = rng.uniform(-s / 2, s / 2, size=(E, n, 2))
    th = np.deg2rad(rng.uniform(0.0, 360.0, size=(E, n, 1)))
    return np.concatenate([xy, th], axis=2).astype(np.float32)


def square_h(E, n):
    """Fixed square side from the GA's initial rule sqrt((0.317 + 0.206/sqrt(n)) n sqrt(1.1))."""
    h0 = np.sqrt((0.317 + 0.206 / np.sqrt(n)) * n * np.sqrt(1.1))
    h = np.zeros((E, 3), dtype=np.float32)
    h[:, 0] = h0
    return h
