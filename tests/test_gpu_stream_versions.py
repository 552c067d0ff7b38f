"""GPU: version-parallel windows of IncrementalBFS.apply_stream.

Without per-batch repair counters, apply_stream answers every batch but the
last with one bit-parallel BFS per window over the window's graph versions,
then commits the window as one merged batch.  After every batch the distances
(checked through the digest) must be the ones applying the batches one at a
time gives, and after the call the graph (vertices, arcs, rows, version
count), the distances, the reachable count and the last batch's repair
counters must be the same too.  Windows of 1 to 256 batches cover every word
count of the kernel (1, 2, 4 and 8 words of version bits per vertex).
"""
import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph
from tests.helpers import messy_stream
from tests.helpers import splitmix_digest as digest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import velographx_b200 as vx  # noqa: E402
import workloads as w  # noqa: E402


def oracle_replay(edges, V, root, src, dst, add, off, directed=False, pre=None):
    """The reference's IncrementalBFS.apply after every batch, and its
    recompute() on the same graph: (graph, bfs, apply digests, recompute
    digests).  The two differ only where the reference's undirected graph has
    let an in-row diverge from its out-row (after its automatic row
    compaction), which the device's single adjacency cannot do; the device
    then gives the recompute distances."""
    og = OracleGraph(V, directed)
    og.bulk_load_edges(edges)
    ob = OracleBFS(og, root)
    if pre is not None:
        ob.apply(*pre)
    digs, fresh = [], []
    for t in range(len(off) - 1):
        lo, hi = int(off[t]), int(off[t + 1])
        ob.apply(src[lo:hi], dst[lo:hi], add[lo:hi])
        digs.append(digest(ob.distances()))
        fresh.append(digest(OracleBFS(og, root).distances()))
    return og, ob, digs, fresh


def check_digests(got, exp, fresh):
    """Every batch equals the reference's recompute, and its apply wherever
    the reference agrees with itself."""
    got = [int(x) for x in got]
    assert [t for t in range(len(got)) if got[t] != fresh[t]] == []
    assert [t for t in range(len(got)) if exp[t] == fresh[t] and got[t] != exp[t]] == []


def counters(b):
    """The reference's observable counters (the affected count only when no
    fallback cut the detection short)."""
    s = b.stats()
    full = s["last_used_full_recompute"]
    return (s["reachable_count"], s["last_deletion_candidates"], full,
            None if full else s["last_affected_vertices"])


def self_consistent(og, exp, fresh):
    """The reference agreed with itself on this stream: apply equals
    recompute after every batch, and every in-row equals its out-row."""
    return exp == fresh and all(sorted(og.neighbors(u)) == sorted(og.in_neighbors(u))
                                for u in range(og.vertex_count))


def check_final(g, b, og, ob, root, seed, consistent):
    """Graph and object state after the call; distances and counters against
    the reference's apply when the reference agrees with itself, else the
    distances against its recompute."""
    if not consistent:
        assert np.array_equal(b.distances_array(), OracleBFS(og, root).distances())
    else:
        assert np.array_equal(b.distances_array(), ob.distances())
        s = b.stats()
        r, c, a, full = ob.stats()
        assert s["reachable_count"] == r
        assert s["last_deletion_candidates"] == c
        assert s["last_used_full_recompute"] == bool(full)
        if not full:
            assert s["last_affected_vertices"] == a
    assert g.vertex_count == og.vertex_count
    assert g.edge_count_directed() == og.edge_count_directed()
    assert g.version == og.version
    for u in np.random.default_rng(seed).integers(0, og.vertex_count, 60).tolist():
        assert sorted(g.neighbors(u)) == sorted(og.neighbors(u)), u


@pytest.mark.parametrize("window", [1, 5, 32, 64, 100, 256])
@pytest.mark.parametrize("seed,grow", [(1, 0), (2, 37)])
def test_windows_match_oracle_after_every_batch(window, seed, grow):
    V = 1 << 12
    edges = w.rmat_edges(12, 8, seed=seed)
    root = w.max_degree_root(edges, V)
    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.choice([0, 1, 7, 40, 300, 2000], size=300, p=[.05, .1, .25, .3, .2, .1])]
    src, dst, add, off = messy_stream(edges, V, sizes, seed + 10, grow)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, root)
    b.set_stream_window(window)
    digs, _ = b.apply_stream(src, dst, add, off, digests=True)
    og, ob, exp, fresh = oracle_replay(edges, V, root, src, dst, add, off)
    check_digests(digs, exp, fresh)
    check_final(g, b, og, ob, root, seed, self_consistent(og, exp, fresh))


def test_toggled_edges_and_rows_changed_before_the_stream():
    """Edges added, removed and re-added within and across batches, on a
    graph whose rows already carry delta entries and tombstones."""
    V = 1 << 11
    edges = w.rmat_edges(11, 8, seed=21)
    root = w.max_degree_root(edges, V)
    e = edges[edges[:, 0] != edges[:, 1]]
    rng = np.random.default_rng(22)
    pre_n = 3000
    pre = (np.concatenate([e[:pre_n // 2, 0], rng.integers(0, V, pre_n // 2).astype(np.uint32)]),
           np.concatenate([e[:pre_n // 2, 1], rng.integers(0, V, pre_n // 2).astype(np.uint32)]),
           np.concatenate([np.zeros(pre_n // 2, np.uint8), np.ones(pre_n // 2, np.uint8)]))
    pool = np.concatenate([e[pre_n // 2: pre_n // 2 + 40], e[:40],
                           np.stack([pre[0][-40:], pre[1][-40:]], 1)])  # live, tombstoned, delta edges
    src, dst, add, off = [], [], [], [0]
    for t in range(90):
        k = int(rng.integers(0, 30))
        pick = pool[rng.integers(0, len(pool), k)]
        flip = rng.random(k) < 0.5
        src.append(np.where(flip, pick[:, 1], pick[:, 0]).astype(np.uint32))
        dst.append(np.where(flip, pick[:, 0], pick[:, 1]).astype(np.uint32))
        add.append(rng.integers(0, 2, k).astype(np.uint8))
        off.append(off[-1] + k)
    src, dst, add = np.concatenate(src), np.concatenate(dst), np.concatenate(add)
    off = np.array(off, np.uint64)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, root)
    b.apply_arrays(*pre)
    b.set_stream_window(16)
    digs, _ = b.apply_stream(src, dst, add, off, digests=True)
    og, ob, exp, fresh = oracle_replay(edges, V, root, src, dst, add, off, pre=pre)
    check_digests(digs, exp, fresh)
    check_final(g, b, og, ob, root, 23, self_consistent(og, exp, fresh))


def test_source_out_of_range_at_construction_stays_unreachable():
    """The reference's quirk: a source past the vertex count when the BFS
    object is made is never reached, even after the graph grows past it."""
    V = 1 << 10
    edges = w.rmat_edges(10, 8, seed=31)
    root = V + 3
    src = np.array([V + 3, 5, V + 9, 1], np.uint32)
    dst = np.array([7, V + 3, 2, V + 3], np.uint32)
    add = np.ones(4, np.uint8)
    off = np.array([0, 1, 2, 3, 3, 4], np.uint64)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, root)
    digs, _ = b.apply_stream(src, dst, add, off, digests=True)
    og, ob, exp, fresh = oracle_replay(edges, V, root, src, dst, add, off)
    assert [int(x) for x in digs] == exp
    assert b.reachable_count == 0
    check_final(g, b, og, ob, root, 32, True)


@pytest.mark.parametrize("scale,window", [(16, 64), (18, 32)])
def test_windows_match_one_batch_at_a_time_path(scale, window):
    """Lognormal batch sizes on R-MAT graphs whose hub rows (2,048+ and
    4,096+ arcs at scale 18) go through the grid-wide pull and push passes."""
    V = 1 << scale
    edges = w.rmat_edges(scale, 16, seed=5 + scale)
    root = w.max_degree_root(edges, V)
    sizes = w.lognormal_sizes(150, median=300, sigma=2.0, hi=30_000, seed=6 + scale)
    st = w.mixed_stream(edges, V, sizes, 0.8, seed=7 + scale)
    off = st.offsets.astype(np.uint64)
    ga, gb = vx.Graph(V, False), vx.Graph(V, False)
    ga.bulk_load_edges(edges)
    gb.bulk_load_edges(edges)
    ba, bb = vx.IncrementalBFS(ga, root), vx.IncrementalBFS(gb, root)
    ba.set_stream_window(window)
    digs, _ = ba.apply_stream(st.src, st.dst, st.add, off, digests=True)
    for t in range(st.batches):
        bb.apply_arrays(*st.batch(t))
        assert int(digs[t]) == bb.digest(), f"batch {t}"
    assert np.array_equal(ba.distances_array(), bb.distances_array())
    assert counters(ba) == counters(bb)
    assert ga.edge_count_directed() == gb.edge_count_directed()
    assert ga.version == gb.version and ga.vertex_count == gb.vertex_count


def test_window_zero_is_the_update_launch_and_both_agree():
    V = 1 << 13
    edges = w.rmat_edges(13, 8, seed=41)
    root = w.max_degree_root(edges, V)
    src, dst, add, off = messy_stream(edges, V, [50, 700, 3, 2500, 0, 90, 1200, 5, 5, 400], 42, grow=20)
    out = []
    for window in (0, 3, 64):
        g = vx.Graph(V, False)
        g.bulk_load_edges(edges)
        b = vx.IncrementalBFS(g, root)
        b.set_stream_window(window)
        digs, _ = b.apply_stream(src, dst, add, off, digests=True)
        out.append(([int(x) for x in digs], counters(b), g.edge_count_directed(), g.version, g.vertex_count,
                    b.distances_array().tobytes()))
    assert out[0] == out[1] == out[2]
