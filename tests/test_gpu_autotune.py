"""GPU: the library's autotuner (vx_bfs_autotune) picks one of its candidate
(alpha, beta, large_row) settings, leaves it applied to the BFS object, and
every result stays exact: the object's own distances after tuning, later
recomputes, and repairs of an update stream (against the oracle's CSR BFS and
a fresh full BFS)."""
import numpy as np
import pytest

import workloads as w
from tests.test_gpu_scale import oracle_bfs

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")


def test_autotune_applies_its_choice_and_stays_exact():
    V = 1 << 17
    e = w.rmat_edges(17, seed=171)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    root = w.max_degree_root(e, V)
    b = vx.IncrementalBFS(g, root)
    before = b.distances_array()
    chosen = b.autotune(w.non_isolated_roots(e, V, 3, seed=172))
    assert chosen["alpha"] in (4.0, 14.0, 40.0, 120.0) and chosen["beta"] in (8.0, 24.0, 96.0)
    assert chosen["large_row"] in (512, 1024, 4096) and chosen["mean_ms"] > 0
    assert b.tuning() == (chosen["alpha"], chosen["beta"], chosen["large_row"])
    assert np.array_equal(b.distances_array(), before)
    assert np.array_equal(before, oracle_bfs(e, V, root, False))
    st = w.mixed_stream(e, V, [4000] * 4, 0.7, seed=173)
    for t in range(st.batches):
        b.apply_arrays(*st.batch(t))
        fresh = vx.IncrementalBFS(g, root)
        assert np.array_equal(b.distances_array(), fresh.distances_array()), t
    b.recompute()
    assert np.array_equal(b.distances_array(), vx.IncrementalBFS(g, root).distances_array())


def test_autotune_rejects_bad_roots():
    g = vx.Graph(16, False)
    g.bulk_load_edges(np.array([[0, 1], [1, 2]], np.uint32))
    b = vx.IncrementalBFS(g, 0)
    with pytest.raises(IndexError):
        b.autotune(np.array([99], np.uint32))
    with pytest.raises(ValueError):
        b.autotune(np.array([], np.uint32))
