"""GPU: consolidate_to_csr_snapshot (include/velographx/storage/consolidation.hpp:
132-163) on the device: after a stream of updates the snapshot holds exactly
the source's logical graph (every row, the edge count, the vertex count and
direction) as a fresh compact CSR with version 1, equal to the reference's
snapshot of the same state, and the source is left as it was (overlay,
version, rows).  The device neighbour-scan probe visits every live arc."""
import numpy as np
import pytest

from oracle import OracleGraph
from oracle.replay import best_kind

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")


@pytest.mark.parametrize("directed", [False, True])
def test_snapshot_equals_logical_graph_and_leaves_source(directed):
    rng = np.random.default_rng(71 + directed)
    V = 500
    e = rng.integers(0, V, size=(3000, 2), dtype=np.uint32)
    og = OracleGraph(V, directed, best_kind())
    og.bulk_load_edges(e)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    for _ in range(8):
        n = 300
        s = rng.integers(0, V + 10, size=n, dtype=np.uint32)
        d = rng.integers(0, V, size=n, dtype=np.uint32)
        a = (rng.random(n) < 0.6).astype(np.uint8)
        pick = rng.integers(0, e.shape[0], size=100)
        s[:100], d[:100], a[:100] = e[pick, 0], e[pick, 1], 0
        og.apply(s, d, a)
        g.apply_arrays(s, d, a)
    before = (g.version, g.delta_edge_count(), g.is_compact(), g.edge_count_directed())
    rows = [g.neighbors(u) for u in range(g.vertex_count)]
    snap = vx.consolidate_to_csr_snapshot(g)
    h = snap["graph"]
    assert (g.version, g.delta_edge_count(), g.is_compact(), g.edge_count_directed()) == before
    assert [g.neighbors(u) for u in range(g.vertex_count)] == rows
    assert h.vertex_count == og.vertex_count and h.directed == directed
    assert h.version == 1 and h.is_compact() and h.delta_edge_count() == 0
    assert h.edge_count_directed() == og.edge_count_directed() == snap["directed_edges"]
    assert [h.neighbors(u) for u in range(h.vertex_count)] == [og.neighbors(u) for u in range(og.vertex_count)]
    assert snap["source_storage_bytes"] == g.storage_bytes()
    assert snap["consolidated_storage_bytes"] == h.storage_bytes()
    assert vx.neighbor_scan_ns(g) > 0 and vx.neighbor_scan_ns(h) > 0


def test_snapshot_of_a_large_graph_runs_bfs_identically():
    import workloads as w

    V = 1 << 18
    e = w.rmat_edges(18, seed=181)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    st = w.mixed_stream(e, V, [20_000] * 5, 0.6, seed=182)
    for t in range(st.batches):
        g.apply_arrays(*st.batch(t))
    h = vx.consolidate_to_csr_snapshot(g)["graph"]
    root = w.max_degree_root(e, V)
    assert np.array_equal(vx.IncrementalBFS(g, root).distances_array(), vx.IncrementalBFS(h, root).distances_array())
    assert h.edge_count_directed() == g.edge_count_directed()
