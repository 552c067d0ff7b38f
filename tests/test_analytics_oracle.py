"""CPU: the restated maintained components and unit-weight SSSP
(oracle/analytics_ref.py, "port") against the unmodified reference's
IncrementalComponents and IncrementalSSSP (oracle/_ref) on random streams
with growth, self-loops, repeated ops and direct graph mutations."""
import numpy as np
import pytest

from oracle import OracleGraph, available
from oracle.analytics_ref import SSSP, Components, canonical

needs_ref = pytest.mark.skipif(not available("reference"), reason="reference build (oracle/_ref) not present")


def random_batch(rng, V, e, n):
    s = rng.integers(0, V + 3, size=n, dtype=np.uint32)
    d = rng.integers(0, V, size=n, dtype=np.uint32)
    a = (rng.random(n) < 0.55).astype(np.uint8)
    k = n // 3
    pick = rng.integers(0, e.shape[0], size=k)
    s[:k], d[:k], a[:k] = e[pick, 0], e[pick, 1], 0
    return s, d, a


@needs_ref
@pytest.mark.parametrize("seed", range(4))
def test_components_port_matches_reference(seed):
    rng = np.random.default_rng(500 + seed)
    V = 60
    e = rng.integers(0, V, size=(70, 2), dtype=np.uint32)
    G = {k: OracleGraph(V, False, k) for k in ("port", "reference")}
    for g in G.values():
        g.bulk_load_edges(e)
    C = {k: Components(G[k]) for k in G}
    for t in range(60):
        s, d, a = random_batch(rng, G["port"].vertex_count, e, int(rng.integers(0, 12)))
        if t % 9 == 4:  # a mutation the components object does not see
            for g in G.values():
                g.apply(s[:2], d[:2], np.ones(min(2, s.size), np.uint8))
            continue
        for c in C.values():
            c.apply(s, d, a)
        n = G["port"].vertex_count + 2
        assert np.array_equal(canonical(C["port"].labels(n)), canonical(C["reference"].labels(n))), t
        assert C["port"].last_repaired_vertices == C["reference"].last_repaired_vertices, t


@needs_ref
@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("source", [0, 70])
def test_sssp_port_matches_reference(directed, source):
    rng = np.random.default_rng(77 + directed + source)
    V = 60
    e = rng.integers(0, V, size=(120, 2), dtype=np.uint32)
    G = {k: OracleGraph(V, directed, k) for k in ("port", "reference")}
    for g in G.values():
        g.bulk_load_edges(e)
    S = {k: SSSP(G[k], source) for k in G}
    for t in range(50):
        s, d, a = random_batch(rng, G["port"].vertex_count + 1, e, int(rng.integers(1, 10)))
        if t % 3:
            a[:] = 1  # insert-only batches take the relaxation path
        for x in S.values():
            x.apply(s, d, a)
        assert np.array_equal(S["port"].distances(), S["reference"].distances()), t
