"""CPU: the oracle restatement (oracle/vx_oracle.c) against the golden vectors made
by the reference itself, the reference's own microcase expectations, and -- when
oracle/_ref is built -- the reference on fresh random streams."""
import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph, available
from tests.golden import scenarios
from tests.helpers import check_record, golden_names, load_golden

ALL = scenarios.all_scenarios()


@pytest.mark.parametrize("name", golden_names())
def test_port_matches_reference_golden(name):
    gold = load_golden(name)
    sc = ALL[name]
    assert scenarios.inputs_digest(sc) == gold["inputs_sha256"], "scenario inputs drifted from the fixture"
    g = OracleGraph(sc["vertices"], sc["directed"], "port")
    if len(sc["edges"]):
        g.bulk_load_edges(sc["edges"])
    b = OracleBFS(g, sc["source"], sc["fraction"])
    prev_v = g.vertex_count
    check_record(gold["records"][0], b.distances(), b.stats(), g.edge_count_directed(), g.version, g.vertex_count,
                 f"{name}[init]", prev_v, sc["fraction"])
    for i, (s, d, a) in enumerate(sc["batches"]):
        prev_v = g.vertex_count
        b.apply(s, d, a)
        check_record(gold["records"][i + 1], b.distances(), b.stats(), g.edge_count_directed(), g.version,
                     g.vertex_count, f"{name}[{i}]", prev_v, sc["fraction"])


def _run(name):
    sc = ALL[name]
    g = OracleGraph(sc["vertices"], sc["directed"], "port")
    g.bulk_load_edges(sc["edges"])
    b = OracleBFS(g, sc["source"], sc["fraction"])
    for s, d, a in sc["batches"]:
        b.apply(s, d, a)
    return g, b


def test_reference_microcase_expectations():
    """Exact expectations written in tests/test_incremental_bfs_deletion.cpp:57-169."""
    U = 0xFFFFFFFF
    g, b = _run("micro_alternate_parent")
    d = b.distances()
    assert d[3] == 2 and d[4] == 3 and b.last_affected_vertices == 0 and not b.last_used_full_recompute
    g, b = _run("micro_support_fixpoint")
    d = b.distances()
    assert list(d[1:5]) == [U] * 4 and b.reachable_count == 1 and b.last_affected_vertices == 4
    g, b = _run("micro_surviving_branch")
    d = b.distances()
    assert d[2] == U and d[3] == 3 and d[4] == 4 and not b.last_used_full_recompute
    g, b = _run("micro_mixed")
    d = b.distances()
    assert d[2] == U and d[3] == 2 and d[4] == 3 and b.reachable_count == 5
    g, b = _run("micro_undirected")
    assert b.distances()[2] == 3
    g, b = _run("micro_final_state")
    d = b.distances()
    assert d[3] == 3 and d[4] == 4
    g, b = _run("micro_fallback")
    assert b.last_used_full_recompute and b.reachable_count == 1
    g, b = _run("micro_out_of_range_source")
    assert b.reachable_count == 0


@pytest.mark.skipif(not available("reference"), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("seed", range(6))
def test_port_matches_reference_live(seed, directed):
    """Random streams with vertex growth, self-loops and interleaved compaction: every
    observable of DynamicGraph and IncrementalBFS agrees with the reference."""
    rng = np.random.default_rng(1000 + seed)
    V = 40
    e = rng.integers(0, V, size=(120, 2), dtype=np.uint32)
    G = {k: OracleGraph(V, directed, k) for k in ("port", "reference")}
    for gg in G.values():
        gg.bulk_load_edges(e)
    frac = [0.05, 0.35, 0.9][seed % 3]
    B = {k: OracleBFS(G[k], 0, frac) for k in G}
    for t in range(120):
        n = int(rng.integers(1, 9))
        s = rng.integers(0, V + (3 if t % 17 == 0 else 0), size=n, dtype=np.uint32)
        d = rng.integers(0, V, size=n, dtype=np.uint32)
        a = (rng.random(n) < 0.5).astype(np.uint8)
        for k in G:
            B[k].apply(s, d, a)
        if t % 13 == 5:  # ensure_vertex between batches (dynamic_graph.hpp:493-500)
            for k in G:
                G[k].ensure_vertex(G[k].vertex_count + 2)
        if t % 11 == 0:
            for k in G:
                G[k].maybe_compact(0.3) if t % 2 else G[k].compact()
        p, r = B["port"], B["reference"]
        assert np.array_equal(p.distances(), r.distances()), t
        assert p.stats() == r.stats(), t
        gp, gr = G["port"], G["reference"]
        assert (gp.vertex_count, gp.version, gp.edge_count_directed(), gp.delta_edge_count(), gp.is_compact(),
                gp.dirty_out_count(), gp.dirty_in_count()) == (
                gr.vertex_count, gr.version, gr.edge_count_directed(), gr.delta_edge_count(), gr.is_compact(),
                gr.dirty_out_count(), gr.dirty_in_count()), t
        assert gp.base_edge_count_directed() == gr.base_edge_count_directed(), t
        for u in range(gp.vertex_count):
            assert gp.neighbors(u) == gr.neighbors(u) and gp.in_neighbors(u) == gr.in_neighbors(u)
            assert gp.compact_neighbors(u) == gr.compact_neighbors(u), (t, u)
            assert gp.compact_in_neighbors(u) == gr.compact_in_neighbors(u), (t, u)


@pytest.mark.skipif(not available("reference"), reason="reference build (oracle/_ref) not present")
def test_port_matches_reference_automatic_maintenance():
    """Enough overlay entries to trigger DynamicGraph's automatic row compaction
    (dynamic_graph.hpp:791-803: >= 65536 delta entries and >= 1% of edges)."""
    rng = np.random.default_rng(5)
    V = 4096
    e = rng.integers(0, V, size=(20000, 2), dtype=np.uint32)
    G = {k: OracleGraph(V, False, k) for k in ("port", "reference")}
    for gg in G.values():
        gg.bulk_load_edges(e)
    B = {k: OracleBFS(G[k], 0, 0.35) for k in G}
    for t in range(6):
        n = 8000
        s = rng.integers(0, V, size=n, dtype=np.uint32)
        d = rng.integers(0, V, size=n, dtype=np.uint32)
        a = (rng.random(n) < 0.8).astype(np.uint8)
        for k in G:
            B[k].apply(s, d, a)
        assert np.array_equal(B["port"].distances(), B["reference"].distances())
        assert B["port"].stats() == B["reference"].stats()
        assert G["port"].delta_edge_count() == G["reference"].delta_edge_count()
        assert G["port"].dirty_out_count() == G["reference"].dirty_out_count()
