"""GPU: the allocation-free BFS entry point (vx_bfs_csr_static).

It exists for callers that cannot call cudaMalloc -- their device memory is
owned by another allocator, or they must not block on the driver's allocator
once running -- and keeps its working memory in one file-scope device array.
Here it is called through the C ABI on device buffers the test owns, twice in
a row, and each result must equal the regular entry point's (IncrementalBFS
on a Graph) bit for bit.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

vx = pytest.importorskip("velographx_b200")
torch = pytest.importorskip("torch")

MAX_VERTICES = 1 << 18


def symmetric_csr(edges, V):
    e = edges[edges[:, 0] != edges[:, 1]].astype(np.uint64)
    k = np.unique(np.concatenate([e[:, 0] << 32 | e[:, 1], e[:, 1] << 32 | e[:, 0]]))
    u = (k >> 32).astype(np.int64)
    off = np.zeros(V + 1, np.uint64)
    np.cumsum(np.bincount(u, minlength=V), out=off[1:])
    return off, (k & 0xFFFFFFFF).astype(np.uint32)


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


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_static_scratch_bfs_rejects_sizes_beyond_its_maximum():
    fn = entry_point()
    d_off = torch.zeros(4, dtype=torch.int64, device="cuda")
    d_col = torch.zeros(4, dtype=torch.int32, device="cuda")
    d_dist = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = fn(d_off.data_ptr(), d_col.data_ptr(), d_off.data_ptr(), d_col.data_ptr(), MAX_VERTICES + 1, 0, 0,
            d_dist.data_ptr(), None, None)
    assert rc == -2 and "262144" in vx.last_error()
