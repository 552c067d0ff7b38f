"""GPU: the allocation-free BFS entry point (vx_bfs_csr_static).

It exists for callers that cannot call cudaMalloc -- their device memory is
owned by another allocator, or they must not block on the driver's allocator
once running -- and keeps its working memory in one file-scope device array.
Here it is called through the C ABI on device buffers the test owns, twice in
a row, and each result must equal the regular entry point's (IncrementalBFS
on a Graph) and the CPU oracle's CSR BFS bit for bit; on an undirected graph
(one CSR passed as out- and in-rows), on a directed one (separate out- and
in-CSRs, which takes the kernel's directed branch) and with a source beyond
the vertex count (all unreachable, nothing reached).  This file is collected
last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

vx = pytest.importorskip("velographx_b200")
torch = pytest.importorskip("torch")

MAX_VERTICES = 1 << 18


def csr(edges, V, directed=False, reverse=False):
    """Deduplicated CSR without self-loops; undirected: both arcs of every
    edge; reverse: the in-rows of a directed graph."""
    e = edges[edges[:, 0] != edges[:, 1]].astype(np.uint64)
    u, v = (e[:, 1], e[:, 0]) if reverse else (e[:, 0], e[:, 1])
    k = u << 32 | v
    if not directed:
        k = np.concatenate([k, v << 32 | u])
    k = np.unique(k)
    off = np.zeros(V + 1, np.uint64)
    np.cumsum(np.bincount((k >> 32).astype(np.int64), minlength=V), out=off[1:])
    return off, (k & 0xFFFFFFFF).astype(np.uint32)


def symmetric_csr(edges, V):
    return csr(edges, V)


def oracle_csr_bfs(off, col, V, root):
    from oracle import load

    lib = load("port")
    dist = np.empty(V, np.uint32)
    assert lib.dll.vxo_csr_bfs(off.ctypes.data_as(C.POINTER(C.c_uint64)), col.ctypes.data_as(C.POINTER(C.c_uint32)),
                               V, root, dist.ctypes.data_as(C.POINTER(C.c_uint32))) == 0
    return dist


def call(fn, out_csr, in_csr, V, root, d_dist, stream):
    """One call through the C ABI; the CSRs are (offsets, cols) torch tensors."""
    reach = C.c_uint64(0)
    rc = fn(out_csr[0].data_ptr(), out_csr[1].data_ptr(), in_csr[0].data_ptr(), in_csr[1].data_ptr(), V,
            int(out_csr[1].numel()), root, d_dist.data_ptr(), stream, C.byref(reach))
    assert rc == 0, vx.last_error()
    return d_dist.cpu().numpy().view(np.uint32).copy(), reach.value


def device_csr(off, col):
    return torch.from_numpy(off.view(np.int64)).cuda(), torch.from_numpy(col.view(np.int32)).cuda()


def entry_point():
    lib = vx.capi()
    fn = lib.vx_bfs_csr_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32, C.c_void_p,
                   C.c_void_p, C.POINTER(C.c_uint64)]
    return fn


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_static_scratch_bfs_matches_regular_entry_point():
    import workloads as w

    V = 1 << 16
    edges = w.rmat_edges(16, seed=16)
    off, col = symmetric_csr(edges, V)
    d_off = torch.from_numpy(off.view(np.int64)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_dist = torch.empty(V, dtype=torch.int32, device="cuda")
    fn = entry_point()
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    roots = [w.max_degree_root(edges, V), int(w.non_isolated_roots(edges, V, 1, seed=9)[0])]
    for root in roots:  # two calls in a row share the static array
        reach = C.c_uint64(0)
        rc = fn(d_off.data_ptr(), d_col.data_ptr(), d_off.data_ptr(), d_col.data_ptr(), V, int(col.size), root,
                d_dist.data_ptr(), stream, C.byref(reach))
        assert rc == 0, vx.last_error()
        got = d_dist.cpu().numpy().view(np.uint32)
        ref = vx.IncrementalBFS(g, root)
        assert np.array_equal(got, ref.distances_array()), f"root {root}"
        assert reach.value == ref.reachable_count
        assert np.array_equal(got, oracle_csr_bfs(off, col, V, root)), f"root {root} (oracle)"


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_static_scratch_bfs_directed_graph_matches_oracle():
    import workloads as w

    V = 1 << 15
    edges = w.rmat_edges(15, seed=151)
    out_c = csr(edges, V, directed=True)
    in_c = csr(edges, V, directed=True, reverse=True)
    d_out, d_in = device_csr(*out_c), device_csr(*in_c)
    d_dist = torch.empty(V, dtype=torch.int32, device="cuda")
    fn = entry_point()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = vx.Graph(V, True)
    g.bulk_load_edges(edges)
    for root in (w.max_degree_root(edges, V), int(w.non_isolated_roots(edges, V, 1, seed=3)[0])):
        got, reach = call(fn, d_out, d_in, V, root, d_dist, stream)
        exp = oracle_csr_bfs(*out_c, V, root)
        assert np.array_equal(got, exp), f"root {root}"
        assert reach == int(np.count_nonzero(exp != 0xFFFFFFFF))
        assert np.array_equal(got, vx.IncrementalBFS(g, root).distances_array())


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_static_scratch_bfs_source_beyond_vertices_is_all_unreachable():
    import workloads as w

    V = 1 << 12
    edges = w.rmat_edges(12, seed=12)
    c = csr(edges, V)
    d = device_csr(*c)
    d_dist = torch.zeros(V, dtype=torch.int32, device="cuda")
    fn = entry_point()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for root in (V, V + 1000):
        got, reach = call(fn, d, d, V, root, d_dist, stream)
        assert reach == 0 and np.all(got == 0xFFFFFFFF)


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_static_scratch_bfs_rejects_sizes_beyond_its_maximum():
    fn = entry_point()
    d_off = torch.zeros(4, dtype=torch.int64, device="cuda")
    d_col = torch.zeros(4, dtype=torch.int32, device="cuda")
    d_dist = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = fn(d_off.data_ptr(), d_col.data_ptr(), d_off.data_ptr(), d_col.data_ptr(), MAX_VERTICES + 1, 0, 0,
            d_dist.data_ptr(), None, None)
    assert rc == -2 and "262144" in vx.last_error()
