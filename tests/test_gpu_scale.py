"""GPU parity at benchmark sizes through size-independent properties, and
bit-exact full BFS against the oracle's CSR BFS at sizes the oracle finishes in
seconds."""
import ctypes as C

import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph
from oracle import load as load_oracle
import workloads as w

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")
U = 0xFFFFFFFF


def simple_arcs(edges, directed):
    e = edges[edges[:, 0] != edges[:, 1]].astype(np.uint64)
    k = e[:, 0] << 32 | e[:, 1]
    if not directed:
        k = np.concatenate([k, e[:, 1] << 32 | e[:, 0]])
    k = np.unique(k)
    return (k >> 32).astype(np.uint32), (k & 0xFFFFFFFF).astype(np.uint32)


def oracle_csr(edges, V, directed):
    u, v = simple_arcs(edges, directed)
    off = np.zeros(V + 1, np.uint64)
    np.cumsum(np.bincount(u, minlength=V), out=off[1:])
    return off, v


def oracle_bfs(edges, V, root, directed, csr=None):
    off, v = csr if csr is not None else oracle_csr(edges, V, directed)
    lib = load_oracle("port")
    dist = np.empty(V, np.uint32)
    rc = lib.dll.vxo_csr_bfs(off.ctypes.data_as(C.POINTER(C.c_uint64)), v.ctypes.data_as(C.POINTER(C.c_uint32)),
                             V, root, dist.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert rc == 0
    return dist


def validate_bfs(dist, edges, root):
    """Graph500-style validation of BFS distances on an undirected edge list."""
    e = edges[edges[:, 0] != edges[:, 1]]
    du = dist[e[:, 0]].astype(np.int64)
    dv = dist[e[:, 1]].astype(np.int64)
    fu, fv = du != U, dv != U
    assert dist[root] == 0
    assert np.all(fu == fv), "an edge joins a reached and an unreached vertex"
    both = fu & fv
    assert np.all(np.abs(du[both] - dv[both]) <= 1), "an edge spans more than one level"
    # every reached vertex except the root has a neighbour one level closer
    V = dist.size
    best = np.full(V, np.iinfo(np.int64).max)
    np.minimum.at(best, e[both, 1], du[both])
    np.minimum.at(best, e[both, 0], dv[both])
    reached = np.flatnonzero(dist != U)
    reached = reached[reached != root]
    assert np.all(best[reached] == dist[reached].astype(np.int64) - 1)


@pytest.mark.parametrize("scale,directed", [(18, False), (16, True)])
def test_full_bfs_matches_oracle(scale, directed):
    V = 1 << scale
    e = w.rmat_edges(scale, seed=scale)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    roots = w.non_isolated_roots(e, V, 4, seed=3).tolist() + [w.max_degree_root(e, V)]
    for r in roots:
        b = vx.IncrementalBFS(g, int(r))
        got = b.distances_array()
        exp = oracle_bfs(e, V, int(r), directed)
        assert np.array_equal(got, exp), f"root {r}"
        assert b.reachable_count == int(np.count_nonzero(exp != U))


def test_grid_high_diameter_full_and_repair():
    e = w.grid_edges(512, 512, long_range_fraction=0.0002, seed=9)
    V = 512 * 512
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, 0)
    assert np.array_equal(b.distances_array(), oracle_bfs(e, V, 0, False))
    lat = e[: 2 * 512 * 511]
    near = lat[(lat[:, 0] // 512 + lat[:, 0] % 512) < 40]
    rng = np.random.default_rng(4)
    for _ in range(5):
        pick = rng.integers(0, near.shape[0], 200)
        s = np.concatenate([near[pick, 0], rng.integers(0, V, 200).astype(np.uint32)])
        d = np.concatenate([near[pick, 1], rng.integers(0, V, 200).astype(np.uint32)])
        a = np.concatenate([np.zeros(200, np.uint8), np.ones(200, np.uint8)])
        b.apply_arrays(s, d, a)
        fresh = vx.IncrementalBFS(g, 0)
        assert np.array_equal(b.distances_array(), fresh.distances_array())
        assert b.reachable_count == fresh.reachable_count


def test_rmat22_config2_repair_equals_recompute():
    """Configuration 2 shape: undirected R-MAT scale 22, batches of 10,000 ops
    (70% uniform insertions, 30% deletions of existing edges).  After every
    batch the repaired distances equal a fresh full BFS bit for bit."""
    scale = 22
    V = 1 << scale
    e = w.rmat_edges(scale, seed=22)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    root = int(w.non_isolated_roots(e, V, 1, seed=5)[0])
    b = vx.IncrementalBFS(g, root)
    validate_bfs(b.distances_array(), e, root)
    st = w.mixed_stream(e, V, [10_000] * 6, 0.7, seed=23)
    for i in range(st.batches):
        s, d, a = st.batch(i)
        b.apply_arrays(s, d, a)
        fresh = vx.IncrementalBFS(g, root)
        got = b.distances_array()
        assert np.array_equal(got, fresh.distances_array()), f"batch {i}"
        assert b.reachable_count == fresh.reachable_count == int(np.count_nonzero(got != U))


@pytest.mark.parametrize("scale,directed,k", [(14, False, 256), (13, True, 33), (12, False, 1)])
def test_multiroot_matches_single_root(scale, directed, k):
    """Every row of the bit-parallel multi-root BFS equals the oracle's BFS from
    that root; roots may repeat or lie outside the graph (all unreachable)."""
    V = 1 << scale
    e = w.rmat_edges(scale, seed=40 + scale)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    rng = np.random.default_rng(scale)
    roots = rng.integers(0, V, size=k).astype(np.uint32)
    if k > 2:
        roots[1] = roots[0]
        roots[2] = V + 5
    m = vx.MultiRootBFS(g, roots)
    m.run()
    got = m.distances_array()
    assert got.shape == (k, V)
    csr = oracle_csr(e, V, directed)
    for r in range(k):
        if roots[r] >= V:
            assert np.all(got[r] == U)
            continue
        exp = oracle_bfs(e, V, int(roots[r]), directed, csr)
        assert np.array_equal(got[r], exp), f"root index {r}"


@pytest.mark.parametrize("scale,k", [(18, 64), (16, 256)])
def test_multiroot_with_hub_rows_repeated_runs(scale, k):
    """Graphs whose hubs (rows of >= 4096 arcs) go through the grid-wide push
    pass; three runs over the same buffers must each equal the oracle."""
    V = 1 << scale
    e = w.rmat_edges(scale, seed=40 + scale)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    roots = w.non_isolated_roots(e, V, k, seed=scale)
    csr = oracle_csr(e, V, False)
    exp = np.stack([oracle_bfs(e, V, int(r), False, csr) for r in roots.tolist()])
    m = vx.MultiRootBFS(g, roots)
    for run in range(3):
        m.run()
        got = m.distances_array()
        bad = [r for r in range(k) if not np.array_equal(got[r], exp[r])]
        assert not bad, f"run {run}: rows {bad[:8]} differ"


def test_multiroot_on_updated_graph():
    """Tombstoned base arcs and delta rows are traversed like the logical graph."""
    V = 1 << 12
    e = w.rmat_edges(12, seed=77)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    st = w.mixed_stream(e, V, [3000, 3000], 0.5, seed=78)
    og = OracleGraph(V, False, "port")
    og.bulk_load_edges(e)
    for i in range(st.batches):
        g.apply_arrays(*st.batch(i))
        og.apply(*st.batch(i))
    roots = np.arange(0, 64, dtype=np.uint32) * 37
    m = vx.MultiRootBFS(g, roots)
    m.run()
    got = m.distances_array()
    for r, root in enumerate(roots.tolist()):
        ob = OracleBFS(og, root)
        assert np.array_equal(got[r], ob.distances()), r
    # a second run over the same buffers gives the same rows
    m.run()
    assert np.array_equal(m.distances_array(), got)
