"""GPU parity: the B200 path (Python module -> C++ mirror -> C ABI -> kernels)
against the reference's golden vectors and the live oracle, bit-exact."""
import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph
from tests.golden import scenarios
from tests.helpers import check_record, golden_names, load_golden

pytestmark = pytest.mark.gpu

vx = pytest.importorskip("velographx_b200")
ALL = scenarios.all_scenarios()


def stats_of(b):
    s = b.stats()
    return (s["reachable_count"], s["last_deletion_candidates"], s["last_affected_vertices"],
            int(s["last_used_full_recompute"]))


def make(sc):
    g = vx.Graph(sc["vertices"], sc["directed"])
    if len(sc["edges"]):
        g.bulk_load_edges(sc["edges"])
    return g, vx.IncrementalBFS(g, sc["source"], sc["fraction"])


@pytest.mark.parametrize("name", golden_names())
def test_gpu_matches_reference_golden(name):
    gold = load_golden(name)
    sc = ALL[name]
    g, b = make(sc)
    check_record(gold["records"][0], b.distances_array(), stats_of(b), g.edge_count_directed(), g.version,
                 g.vertex_count, f"{name}[init]", g.vertex_count, sc["fraction"])
    for i, (s, d, a) in enumerate(sc["batches"]):
        prev_v = g.vertex_count
        b.apply_arrays(s, d, a)
        check_record(gold["records"][i + 1], b.distances_array(), stats_of(b), g.edge_count_directed(), g.version,
                     g.vertex_count, f"{name}[{i}]", prev_v, sc["fraction"])


def test_reference_api_path_microcases():
    """The same microcases through UpdateBatch / .distances (list), as the reference's
    Python users call them."""
    U = vx.IncrementalBFS.unreachable
    g = vx.Graph(5, True)
    g.bulk_load_edges(np.array([[0, 1], [0, 2], [1, 3], [2, 3], [3, 4]], np.uint32))
    b = vx.IncrementalBFS(g, 0, 0.9)
    batch = vx.UpdateBatch()
    batch.remove(0, 1)
    batch.remove(0, 2)
    b.apply(batch)
    assert b.distances == [0, U, U, U, U]
    assert b.reachable_count == 1 and b.last_affected_vertices == 4 and not b.last_used_full_recompute
    # path growth (tests/test_incremental.cpp:20-31)
    g = vx.Graph(5, False)
    batch = vx.UpdateBatch()
    batch.add(0, 1)
    batch.add(1, 2)
    g.apply(batch)
    b = vx.IncrementalBFS(g, 0)
    assert b.distances[2] == 2
    c = vx.UpdateBatch()
    c.add(2, 3)
    b.apply(c)
    assert b.distances[3] == 3
    b.recompute()
    assert b.distances == [0, 1, 2, 3, U]


def test_storage_semantics_directed():
    """tests/test_dynamic.cpp:60-146 on the device graph."""
    d = vx.Graph(6, True)
    d.bulk_load_edges(np.array([[0, 2], [0, 1], [0, 2], [3, 2], [4, 2], [2, 5]], np.uint32))
    assert d.is_compact() and d.edge_count_directed() == 5 and d.version == 1
    assert d.neighbors(0) == [1, 2] and d.in_neighbors(2) == [0, 3, 4] and d.in_neighbors(5) == [2]
    b = vx.UpdateBatch()
    b.remove(0, 2)
    b.add(1, 2)
    b.add(5, 2)
    d.apply(b)
    assert not d.has_edge(0, 2) and d.has_edge(1, 2) and d.has_edge(5, 2)
    assert d.neighbors(0) == [1] and d.in_neighbors(2) == [1, 3, 4, 5] and d.edge_count_directed() == 6
    d.add_edge(0, 2)
    assert d.has_edge(0, 2) and d.in_neighbors(2) == [0, 1, 3, 4, 5]
    before = (d.neighbors(2), d.in_neighbors(2), d.edge_count_directed())
    d.compact()
    assert d.is_compact() and d.delta_edge_count() == 0
    assert (d.neighbors(2), d.in_neighbors(2), d.edge_count_directed()) == before
    d.remove_edge(0, 2)
    d.add_edge(0, 4)
    assert not d.has_edge(0, 2) and d.has_edge(0, 4)
    assert 0 not in d.in_neighbors(2) and 0 in d.in_neighbors(4)
    cnt = d.edge_count_directed()
    d.compact()
    assert d.is_compact() and d.edge_count_directed() == cnt and d.has_edge(0, 4) and not d.has_edge(0, 2)
    d.add_edge(100000, 2)
    assert d.vertex_count == 100001 and d.has_edge(100000, 2) and 100000 in d.in_neighbors(2)


def test_storage_semantics_dirty_rows_and_undirected():
    seed = []
    for i in range(200):
        seed += [(i, 1000 + i), (65536 + i, 67000 + i)]
    s = vx.Graph(131072, True)
    s.bulk_load_edges(np.array(seed, np.uint32))
    assert s.dirty_out_segment_count() == 0 and s.dirty_in_segment_count() == 0
    s.add_edge(10, 50000)
    assert not s.is_compact() and s.dirty_out_segment_count() == 1 and s.dirty_in_segment_count() == 1
    assert 10 in s.in_neighbors(50000)
    s.add_edge(65540, 120000)
    assert s.dirty_out_segment_count() == 2 and s.dirty_in_segment_count() == 2
    cnt = s.edge_count_directed()
    s.compact()
    assert s.is_compact() and s.dirty_out_segment_count() == 0 and s.edge_count_directed() == cnt
    assert s.has_edge(10, 50000) and s.has_edge(65540, 120000)
    u = vx.Graph(4, False)
    b = vx.UpdateBatch()
    b.add(0, 1)
    b.add(1, 2)
    b.add(2, 0)
    u.apply(b)
    assert u.version == 1 and u.has_edge(0, 1) and u.edge_count_directed() == 6
    assert not u.is_compact() and u.delta_edge_count() == 6


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("seed", range(3))
def test_gpu_matches_oracle_live(seed, directed):
    """Random batches with growth, self-loops, repeated ops and interleaved compaction:
    distances, counters and every row agree with the oracle after each batch."""
    rng = np.random.default_rng(77 + seed)
    V = 300
    e = rng.integers(0, V, size=(900, 2), dtype=np.uint32)
    og = OracleGraph(V, directed, "port")
    og.bulk_load_edges(e)
    ob = OracleBFS(og, 0, 0.35)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, 0, 0.35)
    for t in range(60):
        n = int(rng.integers(1, 300))
        s = rng.integers(0, V + (5 if t % 13 == 0 else 0), size=n, dtype=np.uint32)
        d = rng.integers(0, V, size=n, dtype=np.uint32)
        a = (rng.random(n) < 0.55).astype(np.uint8)
        # deletions of existing edges too
        k = n // 3
        pick = rng.integers(0, e.shape[0], size=k)
        s[:k], d[:k], a[:k] = e[pick, 0], e[pick, 1], 0
        ob.apply(s, d, a)
        b.apply_arrays(s, d, a)
        assert np.array_equal(b.distances_array(), ob.distances()), t
        got = stats_of(b)
        exp = ob.stats()
        assert got[0] == exp[0] and got[1] == exp[1] and bool(got[3]) == exp[3], (t, got, exp)
        if not exp[3]:
            assert got[2] == exp[2], (t, got, exp)
        assert g.edge_count_directed() == og.edge_count_directed() and g.version == og.version
        assert g.vertex_count == og.vertex_count
        if t % 20 == 19:
            g.compact()
        if t % 10 == 0:
            for u in rng.integers(0, g.vertex_count, 20):
                assert g.neighbors(int(u)) == og.neighbors(int(u))
                assert g.in_neighbors(int(u)) == og.in_neighbors(int(u))


@pytest.mark.parametrize("directed", [False, True])
def test_boundary_members_match_oracle(directed):
    """ensure_vertex, compact_neighbors / compact_in_neighbors,
    base_edge_count_directed, delta_ratio and storage_bytes
    (dynamic_graph.hpp:493-500, 573-610) against the oracle, with both graphs
    consolidated at the same points; the BFS sees vertices added by
    ensure_vertex exactly as the reference's apply does (bfs.hpp:72-74)."""
    from oracle.replay import best_kind

    kind = best_kind()
    rng = np.random.default_rng(5 + directed)
    V = 200
    e = rng.integers(0, V, size=(700, 2), dtype=np.uint32)
    og = OracleGraph(V, directed, kind)
    og.bulk_load_edges(e)
    ob = OracleBFS(og, 3, 0.35)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, 3, 0.35)
    assert g.storage_bytes() > 0
    for t in range(40):
        if t % 7 == 3:
            grow = g.vertex_count + int(rng.integers(1, 6))
            g.ensure_vertex(grow)
            og.ensure_vertex(grow)
            assert g.vertex_count == og.vertex_count == grow + 1 and g.version == og.version
        n = int(rng.integers(1, 120))
        Vn = g.vertex_count
        s = rng.integers(0, Vn, size=n, dtype=np.uint32)
        d = rng.integers(0, Vn, size=n, dtype=np.uint32)
        a = (rng.random(n) < 0.6).astype(np.uint8)
        k = n // 3
        pick = rng.integers(0, e.shape[0], size=k)
        s[:k], d[:k], a[:k] = e[pick, 0], e[pick, 1], 0
        ob.apply(s, d, a)
        b.apply_arrays(s, d, a)
        assert np.array_equal(b.distances_array(), ob.distances()), t
        assert b.reachable_count == ob.reachable_count
        if t % 9 == 8:
            g.compact()
            og.compact()
        assert g.base_edge_count_directed() == og.base_edge_count_directed(), t
        assert g.delta_edge_count() == og.delta_edge_count(), t
        assert g.delta_ratio() == pytest.approx(g.delta_edge_count() / max(1, g.base_edge_count_directed()))
        if t % 5 == 4:
            for u in range(g.vertex_count):
                assert g.compact_neighbors(u) == og.compact_neighbors(u), (t, u)
                assert g.compact_in_neighbors(u) == og.compact_in_neighbors(u), (t, u)


def test_loaders_and_errors():
    with pytest.raises(ValueError):
        vx.from_numpy_edges(np.zeros((3, 3), np.uint32))
    e = np.array([[0, 1], [1, 2], [2, 2], [1, 0], [5, 3]], np.uint32)
    g = vx.from_numpy_edges(e)
    assert g.vertex_count == 6 and g.version == 1 and g.neighbors(1) == [0, 2] and g.neighbors(3) == [5]
    assert vx.from_numpy_edges(np.zeros((0, 2), np.uint32)).version == 0
    sp = pytest.importorskip("scipy.sparse")
    m = sp.csr_matrix(np.array([[0, 1, 1], [1, 0, 0], [1, 0, 0]]))
    g = vx.from_scipy_csr(m)
    assert g.vertex_count == 3 and g.neighbors(0) == [1, 2] and g.neighbors(2) == [0]
    with pytest.raises(ValueError):
        vx.from_scipy_csr(sp.csr_matrix(np.ones((2, 3))))
    with pytest.raises(ValueError):
        vx.from_scipy_csr(object())
    pa = pytest.importorskip("pyarrow")
    t = pa.table({"src": [0, 1, 2], "dst": [1, 2, 3]})
    g = vx.from_arrow_table(t)
    assert g.neighbors(2) == [1, 3]
    with pytest.raises(ValueError):
        vx.from_arrow_columns(pa.array([0, 1]), pa.array([1]))


def test_capi_direct_calls():
    """The C ABI called directly through ctypes, as a non-Python host would."""
    import ctypes as C

    lib = vx.capi()
    u32p = C.POINTER(C.c_uint32)
    lib.vx_graph_create.argtypes = [C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]
    lib.vx_graph_bulk_load.argtypes = [C.c_void_p, u32p, C.c_size_t]
    lib.vx_bfs_create.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.POINTER(C.c_void_p)]
    lib.vx_bfs_apply.argtypes = [C.c_void_p, u32p, u32p, C.POINTER(C.c_uint8), C.c_size_t]
    lib.vx_bfs_distances.argtypes = [C.c_void_p, u32p, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.vx_bfs_destroy.argtypes = [C.c_void_p]
    lib.vx_graph_destroy.argtypes = [C.c_void_p]
    g = C.c_void_p()
    assert lib.vx_graph_create(4, 0, C.byref(g)) == 0
    uv = np.array([0, 1, 1, 2], np.uint32)
    assert lib.vx_graph_bulk_load(g, uv.ctypes.data_as(u32p), 2) == 0
    b = C.c_void_p()
    assert lib.vx_bfs_create(g, 0, 0.35, C.byref(b)) == 0
    s, d, a = np.array([2], np.uint32), np.array([3], np.uint32), np.array([1], np.uint8)
    assert lib.vx_bfs_apply(b, s.ctypes.data_as(u32p), d.ctypes.data_as(u32p),
                            a.ctypes.data_as(C.POINTER(C.c_uint8)), 1) == 0
    out = np.zeros(4, np.uint32)
    n = C.c_size_t()
    assert lib.vx_bfs_distances(b, out.ctypes.data_as(u32p), 4, C.byref(n)) == 0
    assert n.value == 4 and out.tolist() == [0, 1, 2, 3]
    lib.vx_bfs_destroy(b)
    lib.vx_graph_destroy(g)


@pytest.mark.parametrize("directed", [False, True])
def test_large_batches_use_the_multipass_path(directed):
    """Batches above one cluster's capacity (~90k arcs) take the multi-kernel
    sort path; results must be the same."""
    import workloads as w

    V = 1 << 15
    e = w.rmat_edges(15, seed=31)
    og = OracleGraph(V, directed, "port")
    og.bulk_load_edges(e)
    ob = OracleBFS(og, 0, 0.35)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, 0, 0.35)
    st = w.mixed_stream(e, V, [100_000, 3, 60_000], 0.6, seed=32)
    for i in range(st.batches):
        s, d, a = st.batch(i)
        ob.apply(s, d, a)
        b.apply_arrays(s, d, a)
        assert np.array_equal(b.distances_array(), ob.distances()), i
        assert b.reachable_count == ob.reachable_count
        assert g.edge_count_directed() == og.edge_count_directed()
