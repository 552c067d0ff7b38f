"""GPU: the batched stream path (IncrementalBFS.apply_stream / vx_bfs_apply_stream).

After every batch of a stream, the persistent stream kernel must leave exactly
the state that applying the batches one at a time gives: checked per batch
through the distance digest and the counters, against the oracle on small
graphs and against the one-batch-at-a-time GPU path on larger ones.  The
streams mix insertions, deletions, duplicates and self-loops within batches,
empty batches, vertex growth and a deletion-heavy stretch that triggers the
full-recompute fallback.
"""
import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph
from tests.helpers import fallback_limit, messy_stream
from tests.helpers import splitmix_digest as digest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import velographx_b200 as vx  # noqa: E402
import workloads as w  # noqa: E402


def test_digest_matches_numpy():
    V = 1 << 10
    edges = w.rmat_edges(10, 8, seed=2)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, w.max_degree_root(edges, V))
    assert b.digest() == digest(b.distances_array())


@pytest.mark.parametrize("seed,grow", [(1, 0), (2, 37)])
def test_stream_matches_oracle_after_every_batch(seed, grow):
    V = 1 << 12
    edges = w.rmat_edges(12, 8, seed=seed)
    root = w.max_degree_root(edges, V)
    sizes = [64, 0, 300, 1, 2000, 64, 0, 500, 40, 3000, 7, 128]
    src, dst, add, off = messy_stream(edges, V, sizes, seed + 10, grow)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, root)
    digs, stats = b.apply_stream(src, dst, add, off, digests=True, stats=True)
    og = OracleGraph(V, False)
    og.bulk_load_edges(edges)
    ob = OracleBFS(og, root)
    prev_v = V
    for t in range(len(sizes)):
        lo, hi = int(off[t]), int(off[t + 1])
        ob.apply(src[lo:hi], dst[lo:hi], add[lo:hi])
        d = ob.distances()
        assert int(digs[t]) == digest(d), f"batch {t}: distances differ"
        r, c, a, full = ob.stats()
        assert stats[t, 0] == c, f"batch {t}: candidates {stats[t, 0]} != {c}"
        assert bool(stats[t, 2]) == bool(full), f"batch {t}: full flag"
        if full:
            assert stats[t, 1] > fallback_limit(prev_v, 0.35)
        else:
            assert stats[t, 1] == a, f"batch {t}: affected {stats[t, 1]} != {a}"
        assert stats[t, 3] == (r & 0xFFFFFFFF)
        prev_v = og.vertex_count
    assert np.array_equal(b.distances_array(), ob.distances())
    assert b.reachable_count == ob.reachable_count
    assert g.vertex_count == og.vertex_count
    assert g.edge_count_directed() == og.edge_count_directed()
    assert g.version == og.version
    for u in np.random.default_rng(seed).integers(0, og.vertex_count, 40).tolist():
        assert sorted(g.neighbors(u)) == sorted(og.neighbors(u))


def test_stream_matches_one_batch_at_a_time_path():
    V = 1 << 16
    edges = w.rmat_edges(16, 16, seed=5)
    root = w.max_degree_root(edges, V)
    sizes = w.lognormal_sizes(120, median=500, sigma=2.0, hi=40_000, seed=6)
    st = w.mixed_stream(edges, V, sizes, 0.8, seed=7)
    off = st.offsets.astype(np.uint64)
    ga, gb = vx.Graph(V, False), vx.Graph(V, False)
    ga.bulk_load_edges(edges)
    gb.bulk_load_edges(edges)
    ba, bb = vx.IncrementalBFS(ga, root), vx.IncrementalBFS(gb, root)
    digs, stats = ba.apply_stream(st.src, st.dst, st.add, off, digests=True, stats=True)
    for t in range(st.batches):
        bb.apply_arrays(*st.batch(t))
        s = bb.stats()
        assert int(digs[t]) == bb.digest(), f"batch {t}"
        assert stats[t, 0] == s["last_deletion_candidates"]
        assert bool(stats[t, 2]) == s["last_used_full_recompute"]
        if not s["last_used_full_recompute"]:
            assert stats[t, 1] == s["last_affected_vertices"]
    assert np.array_equal(ba.distances_array(), bb.distances_array())
    assert ga.edge_count_directed() == gb.edge_count_directed()


def test_stream_fallback_and_directed_loop():
    V = 1 << 11
    edges = w.rmat_edges(11, 8, seed=9)
    root = w.max_degree_root(edges, V)
    e = edges[edges[:, 0] != edges[:, 1]]
    # a deletion-heavy batch (most edges removed) forces the full-recompute fallback
    rm = e[: e.shape[0] * 3 // 4]
    src = np.concatenate([rm[:, 0], np.arange(50, dtype=np.uint32)])
    dst = np.concatenate([rm[:, 1], np.arange(50, dtype=np.uint32)[::-1].copy()])
    add = np.concatenate([np.zeros(len(rm), np.uint8), np.ones(50, np.uint8)])
    off = np.array([0, len(rm), len(src)], np.uint64)
    for directed in (False, True):
        g = vx.Graph(V, directed)
        g.bulk_load_edges(edges)
        b = vx.IncrementalBFS(g, root)
        digs, stats = b.apply_stream(src, dst, add, off, digests=True, stats=True)
        og = OracleGraph(V, directed)
        og.bulk_load_edges(edges)
        ob = OracleBFS(og, root)
        for t in range(2):
            lo, hi = int(off[t]), int(off[t + 1])
            ob.apply(src[lo:hi], dst[lo:hi], add[lo:hi])
            assert int(digs[t]) == digest(ob.distances()), (directed, t)
            assert bool(stats[t, 2]) == ob.last_used_full_recompute
        assert np.array_equal(b.distances_array(), ob.distances())


def test_per_phase_and_fused_paths_agree():
    V = 1 << 13
    edges = w.rmat_edges(13, 8, seed=12)
    root = w.max_degree_root(edges, V)
    src, dst, add, off = messy_stream(edges, V, [50, 700, 3, 2500, 0, 90, 1200], 13, grow=20)
    runs = []
    for fused in (False, True):
        g = vx.Graph(V, False)
        g.bulk_load_edges(edges)
        b = vx.IncrementalBFS(g, root)
        b.set_fused(fused)
        rec = []
        for t in range(len(off) - 1):
            lo, hi = int(off[t]), int(off[t + 1])
            b.apply_arrays(src[lo:hi], dst[lo:hi], add[lo:hi])
            s = b.stats()
            rec.append((b.digest(), s["last_deletion_candidates"], s["last_used_full_recompute"],
                        s["reachable_count"], g.edge_count_directed(), g.version))
        runs.append(rec)
    assert runs[0] == runs[1]
