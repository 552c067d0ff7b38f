"""GPU: the graph file formats against the reference.

* load_edge_list (src/io.cpp:23-53), parsed on the device: the same graph
  (vertex count, arc count, every row) or the same error type and message as
  the reference's reader on tricky files, and on an R-MAT scale 14 edge list;
* save_binary (binary_graph.hpp:9-14): byte-identical files to the
  reference's after the same bulk load and update batches;
* load_binary (binary_graph.hpp:15-20): the same vertex count, version, arcs
  and rows as the reference's loader, directed and undirected, and its errors.

The reference is oracle/_ref when built, else the pinned restatement in
oracle/io_ref.py.
"""
import os
import struct
import tempfile

import numpy as np
import pytest

import workloads as w
from oracle import OracleGraph, available
from oracle import io_ref
from tests.test_io_formats import EDGE_LISTS, port_result, reference_result, write_temp

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")
HAVE_REF = available("reference") and os.path.exists(io_ref.TOOL)


def expected_edge_list(path, data, directed):
    return reference_result(path, directed) if HAVE_REF else port_result(data, directed)


def gpu_edge_list(path, directed):
    try:
        g = vx.load_edge_list(path, directed)
    except (RuntimeError, OverflowError) as e:
        return type(e).__name__, str(e)
    V = g.vertex_count
    return V, g.edge_count_directed(), [g.neighbors(u) for u in range(V)]


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("case", range(len(EDGE_LISTS)))
def test_load_edge_list_matches_reference(case, directed):
    data = EDGE_LISTS[case]
    with tempfile.TemporaryDirectory() as tmp:
        path = write_temp(tmp, data)
        assert gpu_edge_list(path, directed) == expected_edge_list(path, data, directed)


@pytest.mark.parametrize("directed", [False, True])
def test_load_edge_list_rmat14(directed):
    e = w.rmat_edges(14, seed=141)
    lines = [f"{u} {v}" if i % 3 else f"  {u}\t{v}  " for i, (u, v) in enumerate(e.tolist())]
    data = ("# R-MAT scale 14\n" + "\n".join(lines) + "\n% end\n").encode()
    with tempfile.TemporaryDirectory() as tmp:
        path = write_temp(tmp, data)
        assert gpu_edge_list(path, directed) == expected_edge_list(path, data, directed)


def graph_pair(directed, seed):
    """The same state on the GPU and in the oracle: a bulk load and a few
    mixed batches, the GPU graph consolidated once midway."""
    rng = np.random.default_rng(seed)
    V = 300
    e = rng.integers(0, V, size=(1200, 2), dtype=np.uint32)
    og = OracleGraph(V, directed, "reference" if HAVE_REF else "port")
    g = vx.Graph(V, directed)
    og.bulk_load_edges(e)
    g.bulk_load_edges(e)
    for t in range(6):
        n = 150
        s = rng.integers(0, V + 20, size=n, dtype=np.uint32)
        d = rng.integers(0, V, size=n, dtype=np.uint32)
        a = (rng.random(n) < 0.6).astype(np.uint8)
        pick = rng.integers(0, e.shape[0], size=n // 3)
        s[: n // 3], d[: n // 3], a[: n // 3] = e[pick, 0], e[pick, 1], 0
        og.apply(s, d, a)
        g.apply_arrays(s, d, a)
        if t == 2:
            g.compact()
    return g, og


@pytest.mark.parametrize("directed", [False, True])
def test_save_binary_bytes_equal_reference(directed):
    g, og = graph_pair(directed, 31 + directed)
    with tempfile.TemporaryDirectory() as tmp:
        mine, theirs = os.path.join(tmp, "gpu.bin"), os.path.join(tmp, "ref.bin")
        vx.save_binary(g, mine)
        if HAVE_REF:
            io_ref.ref_save_binary(og, theirs)
            with open(theirs, "rb") as f:
                expected = f.read()
        else:
            expected = io_ref.binary_bytes(og.vertex_count, [og.neighbors(u) for u in range(og.vertex_count)])
        with open(mine, "rb") as f:
            assert f.read() == expected
        assert not g.is_compact() or g.delta_edge_count() == 0  # saving does not consolidate


@pytest.mark.parametrize("load_directed", [False, True])
@pytest.mark.parametrize("saved_directed", [False, True])
def test_load_binary_matches_reference(saved_directed, load_directed):
    g, og = graph_pair(saved_directed, 47 + saved_directed)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "g.bin")
        vx.save_binary(g, path)
        h = vx.load_binary(path, load_directed)
        if HAVE_REF:
            r = io_ref.ref_load_binary(path, load_directed)
            exp = (r.vertex_count, r.version, r.edge_count_directed(), r.is_compact(),
                   [r.neighbors(u) for u in range(r.vertex_count)])
        else:
            with open(path, "rb") as f:
                _, n, m = struct.unpack("<QQQ", f.read(24))
                pairs = np.frombuffer(f.read(8 * m), np.uint32).reshape(-1, 2)
            keep = pairs if load_directed else pairs[pairs[:, 0] <= pairs[:, 1]]
            r = OracleGraph(n, load_directed, "port")
            r.apply(keep[:, 0], keep[:, 1], np.ones(len(keep), np.uint8))
            r.compact()
            exp = (r.vertex_count, r.version, r.edge_count_directed(), r.is_compact(),
                   [r.neighbors(u) for u in range(r.vertex_count)])
        got = (h.vertex_count, h.version, h.edge_count_directed(), h.is_compact(),
               [h.neighbors(u) for u in range(h.vertex_count)])
        assert got == exp


def test_binary_edge_cases_and_errors():
    with tempfile.TemporaryDirectory() as tmp:
        empty = os.path.join(tmp, "empty.bin")
        with open(empty, "wb") as f:
            f.write(struct.pack("<QQQ", io_ref.MAGIC, 7, 0))
        h = vx.load_binary(empty)
        assert h.vertex_count == 7 and h.version == 0 and h.edge_count_directed() == 0
        only_lower = os.path.join(tmp, "lower.bin")  # undirected load keeps no pair with u > v
        with open(only_lower, "wb") as f:
            f.write(struct.pack("<QQQ", io_ref.MAGIC, 4, 1) + struct.pack("<II", 3, 1))
        h = vx.load_binary(only_lower, False)
        assert h.version == 0 and h.edge_count_directed() == 0
        h = vx.load_binary(only_lower, True)
        assert h.version == 1 and h.neighbors(3) == [1]
        bad = os.path.join(tmp, "bad.bin")
        with open(bad, "wb") as f:
            f.write(struct.pack("<QQQ", 12345, 4, 0))
        with pytest.raises(RuntimeError, match="invalid VeloGraphX binary graph"):
            vx.load_binary(bad)
        short = os.path.join(tmp, "short.bin")
        with open(short, "wb") as f:
            f.write(struct.pack("<QQQ", io_ref.MAGIC, 4, 3) + struct.pack("<II", 0, 1))
        with pytest.raises(RuntimeError, match="truncated graph file"):
            vx.load_binary(short)
        with pytest.raises(RuntimeError, match="cannot open input"):
            vx.load_binary(os.path.join(tmp, "missing.bin"))
        with pytest.raises(RuntimeError, match="unable to open edge-list file"):
            vx.load_edge_list(os.path.join(tmp, "missing.txt"))
