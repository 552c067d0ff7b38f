"""Maintained connected components and unit-weight SSSP on the oracle graph
(test infrastructure only).

* ``kind="reference"`` -- the unmodified reference's IncrementalComponents and
  IncrementalSSSP (include/velographx/incremental/connected_components.hpp,
  sssp.hpp) through oracle/_ref;
* ``kind="port"`` -- a Python restatement of the same procedures over the C
  restatement of the graph (small graphs only), used when the reference is
  not built.

``canonical(labels)`` maps every label to the smallest vertex id carrying it,
so partitions compare as arrays whatever label each implementation picks.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import OracleBFS, OracleGraph, _batch, load

UNREACHABLE_SSSP = (1 << 64) // 4 - 1  # incremental/dijkstra.hpp:14 (UINT64_MAX / 4)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)


def canonical(labels) -> np.ndarray:
    """labels -> smallest vertex id with the same label (entries of
    0xFFFFFFFF, vertices a label vector does not cover, stay as they are)."""
    lab = np.asarray(labels, dtype=np.int64)
    out = lab.copy()
    ok = lab != 0xFFFFFFFF
    if ok.any():
        idx = np.arange(lab.size, dtype=np.int64)
        first = np.full(int(lab[ok].max()) + 1, np.iinfo(np.int64).max)
        np.minimum.at(first, lab[ok], idx[ok])
        out[ok] = first[lab[ok]]
    return out


def _bind():
    lib = load("reference")
    d = lib.dll
    if not getattr(lib, "_an_bound", False):
        d.vxr_cc_create.restype = C.c_void_p
        d.vxr_cc_create.argtypes = [C.c_void_p]
        d.vxr_cc_destroy.argtypes = [C.c_void_p]
        d.vxr_cc_apply.argtypes = [C.c_void_p, _u32p, _u32p, _u8p, C.c_size_t]
        d.vxr_cc_labels.restype = C.c_size_t
        d.vxr_cc_labels.argtypes = [C.c_void_p, _u32p, C.c_size_t]
        d.vxr_cc_last_repaired.restype = C.c_size_t
        d.vxr_cc_last_repaired.argtypes = [C.c_void_p]
        d.vxr_sssp_create.restype = C.c_void_p
        d.vxr_sssp_create.argtypes = [C.c_void_p, C.c_uint32]
        d.vxr_sssp_destroy.argtypes = [C.c_void_p]
        d.vxr_sssp_apply.argtypes = [C.c_void_p, _u32p, _u32p, _u8p, C.c_size_t]
        d.vxr_sssp_recompute.argtypes = [C.c_void_p]
        d.vxr_sssp_distances.restype = C.c_size_t
        d.vxr_sssp_distances.argtypes = [C.c_void_p, _u64p, C.c_size_t]
        lib._an_bound = True
    return d


class Components:
    """IncrementalComponents over an OracleGraph (connected_components.hpp:16-165)."""

    def __init__(self, graph: OracleGraph):
        self.graph = graph
        self.kind = graph.lib.kind
        if self.kind == "reference":
            self.d = _bind()
            self.h = self.d.vxr_cc_create(graph.h)
            if not self.h:
                raise ValueError("IncrementalComponents requires an undirected graph")
        else:
            if graph.directed:
                raise ValueError("IncrementalComponents requires an undirected graph")
            self._rebuild()

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.d.vxr_cc_destroy(h)
            self.h = None

    # ---- restatement (port) ----
    def _find(self, x):
        p = self.parent
        while p[x] != x:
            p[x] = p[p[x]]
            x = p[x]
        return x

    def _unite(self, a, b):
        self._grow()
        a, b = self._find(a), self._find(b)
        if a == b:
            return
        if self.rank[a] < self.rank[b]:
            a, b = b, a
        self.parent[b] = a
        if self.rank[a] == self.rank[b]:
            self.rank[a] += 1

    def _grow(self):
        n = self.graph.vertex_count
        while len(self.parent) < n:
            self.parent.append(len(self.parent))
            self.rank.append(0)

    def _rebuild(self):
        n = self.graph.vertex_count
        self.parent, self.rank = list(range(n)), [0] * n
        for u in range(n):
            for v in self.graph.neighbors(u):
                self._unite(u, v)
        self.last = n

    def apply(self, src, dst, add) -> None:
        s, d, a = _batch(src, dst, add)
        if self.kind == "reference":
            self.d.vxr_cc_apply(self.h, s.ctypes.data_as(_u32p), d.ctypes.data_as(_u32p), a.ctypes.data_as(_u8p),
                                s.size)
            return
        if s.size == 0:
            self.last = 0
            return
        final = {}
        for i in range(s.size - 1, -1, -1):  # last op per undirected edge, self-loops skipped
            u, v = int(s[i]), int(d[i])
            if u == v:
                continue
            key = (min(u, v), max(u, v))
            if key not in final:
                final[key] = bool(a[i])
        n_old = len(self.parent)
        roots = set()
        for (u, v), ad in final.items():
            if not ad and u < n_old and v < n_old and self.graph.has_edge(u, v):
                roots.add(self._find(u))
                roots.add(self._find(v))
        affected = [False] * n_old
        self.last = 0
        if roots:
            for v in range(n_old):
                if self._find(v) in roots:
                    affected[v] = True
                    self.last += 1
        self.graph.apply(s, d, a)
        self._grow()
        affected += [False] * (len(self.parent) - n_old)
        if roots:
            for v in range(len(affected)):
                if affected[v]:
                    self.parent[v], self.rank[v] = v, 0
            for u in range(len(affected)):
                if affected[u]:
                    for v in self.graph.neighbors(u):
                        if v < len(affected) and affected[v]:
                            self._unite(u, v)
        for (u, v), ad in final.items():
            if ad and u < len(self.parent) and v < len(self.parent) and self.graph.has_edge(u, v):
                self._unite(u, v)

    def labels(self, n: int) -> np.ndarray:
        """component(v) for v < n (0xFFFFFFFF where it is out of range)."""
        out = np.full(n, 0xFFFFFFFF, np.uint32)
        if self.kind == "reference":
            self.d.vxr_cc_labels(self.h, out.ctypes.data_as(_u32p), n)
        else:
            for v in range(min(n, len(self.parent))):
                out[v] = self._find(v)
        return out

    @property
    def last_repaired_vertices(self) -> int:
        return self.d.vxr_cc_last_repaired(self.h) if self.kind == "reference" else self.last


class SSSP:
    """IncrementalSSSP over an OracleGraph (sssp.hpp:14-69), unit weights."""

    def __init__(self, graph: OracleGraph, source: int):
        self.graph = graph
        self.kind = graph.lib.kind
        if self.kind == "reference":
            self.d = _bind()
            self.h = self.d.vxr_sssp_create(graph.h, source)
        else:
            self.bfs = OracleBFS(graph, source, 2.0)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.d.vxr_sssp_destroy(h)
            self.h = None

    def apply(self, src, dst, add) -> None:
        s, d, a = _batch(src, dst, add)
        if self.kind == "reference":
            self.d.vxr_sssp_apply(self.h, s.ctypes.data_as(_u32p), d.ctypes.data_as(_u32p), a.ctypes.data_as(_u8p),
                                  s.size)
        elif (a == 0).any():  # any removal: apply, then recompute (sssp.hpp:21-27)
            self.graph.apply(s, d, a)
            self.bfs.recompute()
        else:
            self.bfs.apply(s, d, a)

    def distances(self) -> np.ndarray:
        if self.kind == "reference":
            n = self.d.vxr_sssp_distances(self.h, None, 0)
            out = np.empty(n, np.uint64)
            if n:
                self.d.vxr_sssp_distances(self.h, out.ctypes.data_as(_u64p), n)
            return out
        d32 = self.bfs.distances().astype(np.uint64)
        d32[d32 == 0xFFFFFFFF] = UNREACHABLE_SSSP
        return d32
