"""GPU: delta rows around the boundaries of the fused commit.

The fused launch commits a single-arc row run on a delta row of at most 7
arcs (an insertion) or 8 arcs (a removal) in one lane, in registers, and
every other run through the warp merge.  These batches walk single rows
across both boundaries, in both directions, with single-arc and multi-arc
runs, vertex growth and re-insertion after removal; after every batch the
rows, the overlay counters and the distances must equal the oracle's.
"""
import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import velographx_b200 as vx  # noqa: E402


def batches_for(rng, hub, others, V):
    """Single-op batches that grow hub's delta row one arc at a time to 12
    arcs, a batch that adds 3 at once, removals one at a time back to empty,
    and mixed batches over several rows."""
    out = []
    order = rng.permutation(others)
    for v in order[:12]:
        out.append(([hub], [int(v)], [1]))
    out.append(([hub] * 3, [int(v) for v in order[12:15]], [1, 1, 1]))
    for v in rng.permutation(order[:15]):
        out.append(([hub], [int(v)], [0]))
    # several rows at once, one arc each, some rows near the boundary again
    for _ in range(6):
        k = int(rng.integers(4, 12))
        s = rng.integers(0, V, k)
        d = rng.integers(0, V + 3, k)  # a few ids past V grow the graph
        a = rng.integers(0, 2, k)
        out.append((s.tolist(), d.tolist(), a.tolist()))
    for v in order[:9]:  # refill past 8, then remove the 8th and 9th
        out.append(([hub], [int(v)], [1]))
    out.append(([hub, hub], [int(order[7]), int(order[8])], [0, 0]))
    out.append(([hub], [int(order[0])], [0]))
    return out


@pytest.mark.parametrize("seed", [0, 1])
def test_delta_rows_cross_lane_and_warp_boundaries(seed):
    rng = np.random.default_rng(seed)
    V = 96
    base = np.array([[i, (i * 7 + 3) % V] for i in range(0, V, 2)], np.uint32)
    base = base[base[:, 0] != base[:, 1]]
    hub = 5
    others = [v for v in range(V) if v != hub and not np.any((base[:, 0] == hub) & (base[:, 1] == v))
              and not np.any((base[:, 1] == hub) & (base[:, 0] == v))]
    g = vx.Graph(V, False)
    g.bulk_load_edges(base)
    b = vx.IncrementalBFS(g, 0)
    og = OracleGraph(V, False)
    og.bulk_load_edges(base)
    ob = OracleBFS(og, 0)
    for t, (s, d, a) in enumerate(batches_for(rng, hub, others, V)):
        s = np.asarray(s, np.uint32)
        d = np.asarray(d, np.uint32)
        a = np.asarray(a, np.uint8)
        b.apply_arrays(s, d, a)
        ob.apply(s, d, a)
        n = og.vertex_count
        assert g.vertex_count == n, t
        for u in range(n):
            assert sorted(g.neighbors(u)) == sorted(og.neighbors(u)), (t, u)
        assert g.edge_count_directed() == og.edge_count_directed(), t
        assert g.delta_edge_count() == og.delta_edge_count(), t
        assert np.array_equal(b.distances_array(), ob.distances()), t
