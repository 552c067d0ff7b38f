"""GPU: the update launch's algorithmic-byte accounting (measurement only)
counts every batch and leaves every result unchanged."""
import numpy as np
import pytest

import workloads as w

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")


def test_accounting_counts_and_changes_nothing():
    V = 1 << 16
    e = w.rmat_edges(16, seed=61)
    st = w.mixed_stream(e, V, [2000] * 6, 0.7, seed=62)
    root = w.max_degree_root(e, V)
    digs = []
    for on in (False, True):
        g = vx.Graph(V, False)
        g.bulk_load_edges(e)
        b = vx.IncrementalBFS(g, root)
        b.set_accounting(on)
        d = []
        for t in range(st.batches):
            b.apply_arrays(*st.batch(t))
            d.append(b.digest())
        digs.append(d)
        if on:
            a = b.accounting()
            assert a["batches"] == st.batches
            assert 0 < a["canonical_arcs"] <= 2 * 2000 * st.batches
            assert a["arcs_scanned"] > 0 and a["vertices_visited"] >= a["canonical_arcs"]
            assert a["delta_entries"] > 0
    assert digs[0] == digs[1]
