"""CPU: the seeded generators are deterministic and have the configured shapes."""
import numpy as np

from velographx_b200 import workloads as w


def test_rmat_deterministic_and_skewed():
    a = w.rmat_edges(12, seed=3)
    b = w.rmat_edges(12, seed=3)
    assert a.shape == (16 << 12, 2) and np.array_equal(a, b)
    assert not np.array_equal(a, w.rmat_edges(12, seed=4))
    deg = np.bincount(a.ravel(), minlength=1 << 12)
    assert deg.max() > 20 * deg.mean()  # heavy-tailed (a = 0.57)
    assert a.max() < (1 << 12)


def test_grid_shape():
    g = w.grid_edges(8, 8, long_range_fraction=0.0)
    assert g.shape == (2 * 8 * 7, 2)
    assert set(map(tuple, g[:3].tolist())) == {(0, 1), (1, 2), (2, 3)}
    g2 = w.grid_edges(64, 64, 0.001)
    assert g2.shape[0] == 2 * 64 * 63 + round(2 * 64 * 63 * 0.001)


def test_streams():
    e = w.rmat_edges(10, seed=1)
    st = w.mixed_stream(e, 1024, [10, 20, 30], 0.7, seed=2)
    assert st.batches == 3 and st.src.size == 60
    s, d, a = st.batch(1)
    assert s.size == 20
    sizes = w.lognormal_sizes(1000)
    assert sizes.min() >= 1 and sizes.max() <= 200_000 and 300 < np.median(sizes) < 800
    roots = w.non_isolated_roots(e, 1024, 16)
    assert roots.size == 16 and len(set(roots.tolist())) == 16
