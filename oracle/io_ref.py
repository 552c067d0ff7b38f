"""The reference's graph file formats (test infrastructure only).

* A Python restatement of the binary graph format
  (include/velographx/io/binary_graph.hpp:9-20) and of the text edge-list
  reader (src/io.cpp:23-53), pinned against the reference by the CPU tests;
* the same entry points of the unmodified reference (oracle/_ref):
  ``ref_save_binary`` and ``ref_load_binary`` in-process through the shim,
  ``ref_load_edge_list`` through ``_ref/ref_io_tool`` in a process of its own
  (oracle/ref_io_tool.cpp says why).

Errors are raised as the reference raises them: ``RuntimeError`` for
std::runtime_error, ``OverflowError`` for std::overflow_error, with the
reference's message.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess

import numpy as np

from .oracle import OracleGraph, load

MAGIC = 0x564758303031
_SPACE = b" \t\n\v\f\r"
_U64_MAX = (1 << 64) - 1
TOOL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "ref_io_tool")


def binary_bytes(vertex_count: int, rows) -> bytes:
    """save_binary (binary_graph.hpp:9-14): u64 magic, u64 vertex count, u64 arc
    count, then (u32 u, u32 v) for every arc, rows in vertex order."""
    m = sum(len(r) for r in rows)
    out = [struct.pack("<QQQ", MAGIC, vertex_count, m)]
    for u, r in enumerate(rows):
        if len(r):
            a = np.empty((len(r), 2), np.uint32)
            a[:, 0] = u
            a[:, 1] = r
            out.append(a.tobytes())
    return b"".join(out)


def _read_u64(s: bytes, i: int):
    """istream >> uint64_t in the C locale: whitespace, optional sign, digits;
    a magnitude past 2^64 - 1 fails; '-' negates modulo 2^64."""
    n = len(s)
    while i < n and s[i] in _SPACE:
        i += 1
    neg = False
    if i < n and s[i] in b"+-":
        neg = s[i] == ord("-")
        i += 1
    j = i
    while j < n and 48 <= s[j] <= 57:
        j += 1
    if j == i:
        return None, j
    v = int(s[i:j])
    if v > _U64_MAX:
        return None, j
    return ((-v) & _U64_MAX) if neg else v, j


def parse_edge_list(data: bytes, directed: bool = False):
    """load_edge_list (src/io.cpp:23-53) restated: returns (vertex_count, arcs)
    of the CsrGraph it builds (src/csr_graph.cpp:7-42: self-loops dropped,
    undirected edges both ways, arcs sorted and unique)."""
    edges = []
    lines = data.split(b"\n")
    for k, line in enumerate(lines, start=1):
        if k == len(lines) and line == b"":
            break  # getline yields no line after a final newline
        i = 0
        while i < len(line) and line[i] in _SPACE:
            i += 1
        if i == len(line) or line[i] in b"#%":
            continue
        u, i = _read_u64(line, i)
        v = None
        if u is not None:
            v, i = _read_u64(line, i)
        if u is None or v is None:
            raise RuntimeError(f"malformed edge list at line {k}")
        if u > 0xFFFFFFFF or v > 0xFFFFFFFF:
            raise OverflowError(f"vertex id exceeds uint32 range at line {k}")
        while i < len(line) and line[i] in _SPACE:
            i += 1
        if i < len(line):
            raise RuntimeError(f"unexpected trailing data at line {k}")
        edges.append((u, v))
    arcs = set()
    vmax = -1
    for u, v in edges:
        if u == v:
            continue
        arcs.add((u, v))
        if not directed:
            arcs.add((v, u))
        vmax = max(vmax, u, v)
    return vmax + 1, sorted(arcs)


# ---- the unmodified reference (oracle/_ref) --------------------------------

def _ref():
    lib = load("reference")
    d = lib.dll
    if not getattr(lib, "_io_bound", False):
        d.vxr_save_binary.restype = C.c_int
        d.vxr_save_binary.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t]
        d.vxr_load_binary.restype = C.c_void_p
        d.vxr_load_binary.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_size_t]
        lib._io_bound = True
    return d


def ref_save_binary(g: OracleGraph, path: str) -> None:
    assert g.lib.kind == "reference"
    msg = C.create_string_buffer(512)
    if _ref().vxr_save_binary(g.h, path.encode(), msg, 512) != 0:
        raise RuntimeError(msg.value.decode())


def ref_load_binary(path: str, directed: bool = False) -> OracleGraph:
    msg = C.create_string_buffer(512)
    h = _ref().vxr_load_binary(path.encode(), int(directed), msg, 512)
    if not h:
        raise RuntimeError(msg.value.decode())
    g = OracleGraph.__new__(OracleGraph)
    g.lib = load("reference")
    g.directed = directed
    g.h = h
    return g


def ref_load_edge_list(path: str, directed: bool = False):
    """(vertex_count, arc count, rows) of the reference's CsrGraph."""
    out = subprocess.run([TOOL, path, str(int(directed))], capture_output=True, text=True, check=True).stdout
    head, _, rest = out.partition("\n")
    if head.startswith("overflow_error "):
        raise OverflowError(head[len("overflow_error "):])
    if head.startswith("runtime_error "):
        raise RuntimeError(head[len("runtime_error "):])
    _, V, m = head.split()
    lines = rest.split("\n")
    rows = [[int(x) for x in lines[u].split()] for u in range(int(V))]
    return int(V), int(m), rows
