"""Size classes of ragged batches (host logic, no GPU)."""
import numpy as np
import pytest

from packing_b200.relax import CLASS_EDGES, CLASS_TABLE, size_classes


def test_classes_cover_a_largest_first_order():
    rng = np.random.default_rng(5)
    sizes = np.sort(np.round(np.exp(rng.uniform(np.log(1), np.log(1024), 5000))).astype(int))[::-1]
    cls = size_classes(sizes)
    assert cls[0].start == 0 and sum(c.count for c in cls) == len(sizes)
    for a, b in zip(cls, cls[1:]):
        assert a.start + a.count == b.start and a.n_max > b.n_max
    for c in cls:
        part = sizes[c.start:c.start + c.count]
        assert c.n_max == part.max()
        edge = min(e for e in CLASS_EDGES if e >= c.n_max)
        lower = max([e for e in CLASS_EDGES if e < edge], default=0)
        assert (part > lower).all()
        assert c.threads == dict(CLASS_TABLE)[edge] and c.threads % 32 == 0 and 32 <= c.threads <= 256
        assert 8 * c.threads >= c.n_max - 1      # the kernel's near-list rule


def test_class_edge_cases():
    assert size_classes([]) == []
    assert [c.threads for c in size_classes([200, 200, 5])] == [256, 32]
    assert [(c.n_max, c.count, c.threads) for c in size_classes([161, 160, 121, 120, 81, 80])] == \
        [(161, 1, 256), (160, 2, 192), (120, 2, 128), (80, 1, 96)]
    with pytest.raises(ValueError):
        size_classes([5, 200])
    with pytest.raises(ValueError):
        size_classes([2000])
