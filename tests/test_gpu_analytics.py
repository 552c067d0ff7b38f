"""GPU: the maintained connected components and unit-weight SSSP on the
device graph against the reference's IncrementalComponents and
IncrementalSSSP (include/velographx/incremental/connected_components.hpp,
sssp.hpp) after every batch: the partition (labels compared through the
smallest id of each class), last_repaired_vertices, and the 64-bit
distances.  The reference is oracle/_ref when built, else the pinned
restatement (oracle/analytics_ref.py)."""
import numpy as np
import pytest

import workloads as w
from oracle import OracleGraph
from oracle.analytics_ref import SSSP, UNREACHABLE_SSSP, Components, canonical
from oracle.replay import best_kind
from tests.test_analytics_oracle import random_batch

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")


def gpu_labels(cc, n):
    lab = np.full(n, 0xFFFFFFFF, np.int64)
    got = cc.labels_array()
    lab[: min(n, got.size)] = got[:n]
    return lab


@pytest.mark.parametrize("seed", range(3))
def test_components_match_reference_every_batch(seed):
    rng = np.random.default_rng(900 + seed)
    V = 400
    e = rng.integers(0, V, size=(420, 2), dtype=np.uint32)  # sparse: many components
    og = OracleGraph(V, False, best_kind())
    og.bulk_load_edges(e)
    oc = Components(og)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    cc = vx.IncrementalComponents(g)
    n = V + 2
    assert np.array_equal(gpu_labels(cc, n), canonical(oc.labels(n)))
    assert cc.last_repaired_vertices == oc.last_repaired_vertices == V
    for t in range(40):
        s, d, a = random_batch(rng, g.vertex_count, e, int(rng.integers(0, 60)))
        if t % 11 == 7:  # a mutation the components object does not see (as in the reference)
            g.apply_arrays(s[:3], d[:3], np.ones(min(3, s.size), np.uint8))
            og.apply(s[:3], d[:3], np.ones(min(3, s.size), np.uint8))
            continue
        cc.apply_arrays(s, d, a)
        oc.apply(s, d, a)
        n = g.vertex_count + 2
        assert np.array_equal(gpu_labels(cc, n), canonical(oc.labels(n))), t
        assert cc.last_repaired_vertices == oc.last_repaired_vertices, t
        assert g.version == og.version and g.vertex_count == og.vertex_count


def test_components_rmat16_large_batches():
    V = 1 << 16
    e = w.rmat_edges(16, 4, seed=161)  # edge factor 4: a giant component and many small ones
    og = OracleGraph(V, False, best_kind())
    og.bulk_load_edges(e)
    oc = Components(og)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    cc = vx.IncrementalComponents(g)
    st = w.mixed_stream(e, V, [5000] * 4, 0.5, seed=162)
    for t in range(st.batches):
        s, d, a = st.batch(t)
        cc.apply_arrays(s, d, a)
        oc.apply(s, d, a)
        assert np.array_equal(gpu_labels(cc, V), canonical(oc.labels(V))), t
        assert cc.last_repaired_vertices == oc.last_repaired_vertices, t


def test_components_api_semantics():
    """The reference's own microcase (tests/test_incremental_components_deletion.cpp)
    through the Python surface, and its errors."""
    g = vx.Graph(8, False)
    b = vx.UpdateBatch()
    for u, v in ((0, 1), (1, 2), (2, 3), (4, 5), (5, 6)):
        b.add(u, v)
    g.apply(b)
    cc = vx.IncrementalComponents(g)
    assert cc.component(0) == cc.component(3) and cc.component(4) == cc.component(6)
    assert cc.component(0) != cc.component(4)
    d = vx.UpdateBatch()
    d.remove(1, 2)
    cc.apply(d)
    assert cc.component(0) == cc.component(1) and cc.component(2) == cc.component(3)
    assert cc.component(0) != cc.component(2) and cc.last_repaired_vertices == 4
    m = vx.UpdateBatch()
    m.remove(4, 5)
    m.add(1, 2)
    cc.apply(m)
    assert cc.component(0) == cc.component(3) and cc.component(4) != cc.component(5)
    assert cc.component(5) == cc.component(6) and cc.last_repaired_vertices == 3
    cc.apply(vx.UpdateBatch())
    assert cc.last_repaired_vertices == 0
    with pytest.raises(IndexError):
        cc.component(8)
    with pytest.raises(ValueError):
        vx.IncrementalComponents(vx.Graph(4, True))


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("source", [0, 420])
def test_sssp_matches_reference_every_batch(directed, source):
    rng = np.random.default_rng(31 + directed + source)
    V = 400
    e = rng.integers(0, V, size=(1600, 2), dtype=np.uint32)
    og = OracleGraph(V, directed, best_kind())
    og.bulk_load_edges(e)
    osp = SSSP(og, source)
    g = vx.Graph(V, directed)
    g.bulk_load_edges(e)
    sp = vx.IncrementalSSSP(g, source)
    assert vx.IncrementalSSSP.unreachable == UNREACHABLE_SSSP
    for t in range(40):
        s, d, a = random_batch(rng, g.vertex_count + 2, e, int(rng.integers(1, 80)))
        if t % 3:
            a[:] = 1
        b = vx.UpdateBatch()
        for x, y, z in zip(s.tolist(), d.tolist(), a.tolist()):
            b.add(x, y) if z else b.remove(x, y)
        sp.apply(b)
        osp.apply(s, d, a)
        assert np.array_equal(np.asarray(sp.distances, np.uint64), osp.distances()), t
