"""CPU: the Python restatement of the reference's graph file formats
(oracle/io_ref.py) against the unmodified reference (oracle/_ref): the text
edge-list reader on tricky inputs -- comments, blank lines, CRLF, signs, ids at
and past the uint32 range, magnitudes past 2^64, trailing data, no final
newline -- and the binary format's bytes."""
import os
import tempfile

import numpy as np
import pytest

from oracle import OracleGraph, available
from oracle import io_ref

# (file contents, whether the reference materialises it cheaply)
EDGE_LISTS = [
    b"   # comment\n\t% another comment\n0 1\n1 2   \n",
    b"0 1\n1 2\n2 0",
    b"0 1\r\n1 2\r\n",
    b"\n\n5 3\n\n",
    b"+4 -0\n7 7\n",
    b"0\n",
    b"abc def\n",
    b"0 1 junk\n",
    b"4294967296 1\n",
    b"0 1\n1 2 extra\n2 3\n",
    b"1 2\n-1 3\n",
    b"-18446744073709551615 2\n",
    b"18446744073709551616 2\n",
    b"1 2\n3 4\n5\n7 99999999999 x\n",
    b"1\t\t2\n\v3 4\f\n",
    b"1 2 # inline comment\n",
    b"",
    b"# only comments\n%\n",
    b"1,2\n",
    b"0x10 3\n",
    b"3 1\n1 3\n2 2\n",
]


def write_temp(tmp, data: bytes, name="edges.txt") -> str:
    path = os.path.join(tmp, name)
    with open(path, "wb") as f:
        f.write(data)
    return path


def port_result(data, directed):
    """(V, arcs, rows) or (error type name, message) from the restatement."""
    try:
        V, arcs = io_ref.parse_edge_list(data, directed)
    except (RuntimeError, OverflowError) as e:
        return type(e).__name__, str(e)
    rows = [[] for _ in range(V)]
    for u, v in arcs:
        rows[u].append(v)
    return V, len(arcs), rows


def reference_result(path, directed):
    try:
        return io_ref.ref_load_edge_list(path, directed)
    except (RuntimeError, OverflowError) as e:
        return type(e).__name__, str(e)


needs_ref = pytest.mark.skipif(not (available("reference") and os.path.exists(io_ref.TOOL)),
                               reason="reference build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("case", range(len(EDGE_LISTS)))
def test_edge_list_restatement_matches_reference(case, directed):
    data = EDGE_LISTS[case]
    with tempfile.TemporaryDirectory() as tmp:
        ref = reference_result(write_temp(tmp, data), directed)
    assert port_result(data, directed) == ref


@needs_ref
@pytest.mark.parametrize("directed", [False, True])
def test_binary_bytes_restatement_matches_reference(directed):
    rng = np.random.default_rng(9 + directed)
    g = OracleGraph(50, directed, "reference")
    g.bulk_load_edges(rng.integers(0, 50, size=(200, 2), dtype=np.uint32))
    s = rng.integers(0, 60, size=40, dtype=np.uint32)
    d = rng.integers(0, 60, size=40, dtype=np.uint32)
    g.apply(s, d, (rng.random(40) < 0.6).astype(np.uint8))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "g.bin")
        io_ref.ref_save_binary(g, path)
        with open(path, "rb") as f:
            data = f.read()
        rows = [g.neighbors(u) for u in range(g.vertex_count)]
        assert data == io_ref.binary_bytes(g.vertex_count, rows)
        h = io_ref.ref_load_binary(path, directed)
        assert [h.neighbors(u) for u in range(h.vertex_count)] == rows and h.version == 1
