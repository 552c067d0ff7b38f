"""GPU: batches already in device memory (apply_device).

The device entry points read the caller's arrays in place on the graph's
stream.  A stream applied through them must leave, after every batch, the
graph and distances that the host-array entry points leave -- with vertex
growth, with the graph-only entry point, and with one device buffer that is
rewritten on the same stream for every batch (the rewrite is ordered after
the previous call's reads).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import velographx_b200 as vx  # noqa: E402
import workloads as w  # noqa: E402


def vertex_count_after(vcount, s, d):
    m = s != d
    return max(vcount, int(max(s[m].max(initial=0), d[m].max(initial=0))) + 1 if m.any() else vcount)


@pytest.mark.parametrize("directed", [False, True])
def test_device_batches_match_host_batches(directed):
    V = 1 << 12
    edges = w.rmat_edges(12, 8, seed=31)
    root = w.max_degree_root(edges, V)
    sizes = [300, 1, 2000, 0, 750, 64, 4000, 9]
    st = w.mixed_stream(edges, V, sizes, 0.6, seed=32)
    src, dst, add = st.src.copy(), st.dst.copy(), st.add.copy()
    grow = np.random.default_rng(33).integers(0, src.size, 12)
    dst[grow] = V + np.arange(12, dtype=np.uint32)  # new vertices
    gh, gd = vx.Graph(V, directed), vx.Graph(V, directed)
    gh.bulk_load_edges(edges)
    gd.bulk_load_edges(edges)
    bh, bd = vx.IncrementalBFS(gh, root), vx.IncrementalBFS(gd, root)
    cs = torch.cuda.ExternalStream(gd.stream)
    cap = max(sizes)
    # one set of device buffers, rewritten on the graph's stream for every batch
    ds = torch.empty(cap, dtype=torch.int32, device="cuda")
    dd = torch.empty(cap, dtype=torch.int32, device="cuda")
    da = torch.empty(cap, dtype=torch.uint8, device="cuda")
    for t in range(len(sizes)):
        lo, hi = int(st.offsets[t]), int(st.offsets[t + 1])
        s, d, a = src[lo:hi], dst[lo:hi], add[lo:hi]
        n = hi - lo
        with torch.cuda.stream(cs):
            if n:
                ds[:n].copy_(torch.from_numpy(s.view(np.int32)), non_blocking=False)
                dd[:n].copy_(torch.from_numpy(d.view(np.int32)), non_blocking=False)
                da[:n].copy_(torch.from_numpy(a), non_blocking=False)
        vafter = vertex_count_after(gd.vertex_count, s, d)
        bd.apply_device(ds.data_ptr(), dd.data_ptr(), da.data_ptr(), n, vafter)
        bh.apply_arrays(s, d, a)
        assert gd.vertex_count == gh.vertex_count, t
        assert gd.edge_count_directed() == gh.edge_count_directed(), t
        assert gd.version == gh.version, t
        assert np.array_equal(bd.distances_array(), bh.distances_array()), t
        sd, sh = bd.stats(), bh.stats()
        for k in ("reachable_count", "last_deletion_candidates", "last_used_full_recompute"):
            assert sd[k] == sh[k], (t, k)
    for u in np.random.default_rng(34).integers(0, gd.vertex_count, 64).tolist():
        assert sorted(gd.neighbors(u)) == sorted(gh.neighbors(u))


def test_graph_only_device_batches():
    V = 1 << 10
    edges = w.rmat_edges(10, 8, seed=41)
    st = w.mixed_stream(edges, V, [200, 500, 50], 0.5, seed=42)
    gh, gd = vx.Graph(V, False), vx.Graph(V, False)
    gh.bulk_load_edges(edges)
    gd.bulk_load_edges(edges)
    for t in range(st.batches):
        s, d, a = st.batch(t)
        ts = torch.from_numpy(s.view(np.int32)).cuda()
        td = torch.from_numpy(d.view(np.int32)).cuda()
        ta = torch.from_numpy(a).cuda()
        torch.cuda.synchronize()
        gd.apply_device(ts.data_ptr(), td.data_ptr(), ta.data_ptr(), s.size, vertex_count_after(gd.vertex_count, s, d))
        gh.apply_arrays(s, d, a)
        gd.synchronize()
        assert gd.edge_count_directed() == gh.edge_count_directed(), t
        for u in range(0, V, 37):
            assert sorted(gd.neighbors(u)) == sorted(gh.neighbors(u)), (t, u)


def test_repeated_bulk_loads_size_the_graph_exactly():
    """Host edge lists are uploaded on the graph's own stream: graph after graph
    in one process (device memory reused between them), the vertex count after
    a bulk load is max id + 1 and the arc count is the loaded one."""
    base = w.rmat_edges(13, 8, seed=12)
    e = base[base[:, 0] != base[:, 1]]
    expect_arcs = np.unique(np.concatenate([e[:, 0].astype(np.uint64) << 32 | e[:, 1],
                                            e[:, 1].astype(np.uint64) << 32 | e[:, 0]])).size
    V = 1 << 13
    for t in range(12):
        edges = base.copy()  # a fresh host array each time
        g = vx.Graph(V if t % 2 else 16, False)
        g.bulk_load_edges(edges)
        assert g.vertex_count == max(V if t % 2 else 16, int(e.max()) + 1), t
        assert g.edge_count_directed() == expect_arcs, t
        b = vx.IncrementalBFS(g, 0)
        assert b.distances_array().size == g.vertex_count, t


def test_device_batch_vertex_bound_is_checked():
    g = vx.Graph(16, False)
    b = vx.IncrementalBFS(g, 0)
    t = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        b.apply_device(t.data_ptr(), t.data_ptr(), t.data_ptr(), 1, 8)  # below vertex_count
