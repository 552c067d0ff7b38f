"""A defect of the reference, pinned on the CPU so that the device's deviation
from it stays documented and visible.

The reference's undirected DynamicGraph keeps an out-overlay and an
in-overlay.  apply_arc (include/velographx/storage/dynamic_graph.hpp:726-734)
writes the in-overlay entry with the *out* row's base presence
(`delta_in_.set(v, u, present, base_present_out)`).  Once its automatic
maintenance (:791-802, after 65,536 delta entries) has compacted a row on one
side only, that presence is the wrong one for the other side, and an in-row
can stop matching its out-row.  IncrementalBFS::apply reads in-rows for its
support counts and boundary distances (incremental/bfs.hpp:211-220, 261-270)
and out-rows for everything else, so its distances can then differ from its
own recompute() on the same graph.

The device stores one adjacency for an undirected graph, so its in-rows are
its out-rows: after such a batch its distances are the reference's
recompute() distances (tests/test_gpu_stream_versions.py checks both).  This
test replays a stream of duplicates, removals and re-additions through the
reference and asserts the divergence is there; it is skipped when the
reference is not built.
"""
import numpy as np
import pytest

import workloads as w
from oracle import OracleBFS, OracleGraph
from oracle.replay import best_kind
from tests.helpers import messy_stream


def test_reference_in_rows_diverge_and_apply_differs_from_recompute():
    if best_kind() != "reference":
        pytest.skip("oracle/_ref not built")
    V = 1 << 12
    edges = w.rmat_edges(12, 8, seed=1)
    root = w.max_degree_root(edges, V)
    rng = np.random.default_rng(1)
    sizes = [int(x) for x in rng.choice([0, 1, 7, 40, 300, 2000], size=300, p=[.05, .1, .25, .3, .2, .1])]
    src, dst, add, off = messy_stream(edges, V, sizes, 11)
    og = OracleGraph(V, False, "reference")
    og.bulk_load_edges(edges)
    ob = OracleBFS(og, root)
    first_rows = first_dist = None
    for t in range(len(sizes)):
        lo, hi = int(off[t]), int(off[t + 1])
        ob.apply(src[lo:hi], dst[lo:hi], add[lo:hi])
        if first_rows is None and any(sorted(og.neighbors(u)) != sorted(og.in_neighbors(u)) for u in range(V)):
            first_rows = t
        if first_rows is not None and not np.array_equal(ob.distances(), OracleBFS(og, root).distances()):
            first_dist = t
            break
    # this seed: rows first diverge at batch 167 (a deleted base edge re-added
    # after row compaction), the distances at batch 221
    assert first_rows == 167
    assert first_dist == 221
