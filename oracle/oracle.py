"""ctypes bindings for the oracle libraries (see ``oracle/__init__.py``)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
UNREACHABLE = 0xFFFFFFFF
_PATHS = {
    "port": os.path.join(HERE, "liboracle.so"),
    "reference": os.path.join(HERE, "_ref", "libvxref.so"),
}
_PREFIX = {"port": "vxo_", "reference": "vxr_"}
_LIBS: dict[str, C.CDLL] = {}

_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p
_sz = C.c_size_t

_SIGS = {
    "graph_create": (_vp, [_sz, C.c_int]),
    "graph_destroy": (None, [_vp]),
    "graph_vertex_count": (_sz, [_vp]),
    "graph_version": (C.c_uint64, [_vp]),
    "graph_bulk_load": (C.c_int, [_vp, _u32p, _sz]),
    "graph_apply": (C.c_int, [_vp, _u32p, _u32p, _u8p, _sz]),
    "graph_neighbors": (_sz, [_vp, C.c_uint32, _u32p, _sz]),
    "graph_in_neighbors": (_sz, [_vp, C.c_uint32, _u32p, _sz]),
    "graph_has_edge": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "graph_edge_count_directed": (_sz, [_vp]),
    "graph_delta_edge_count": (_sz, [_vp]),
    "graph_is_compact": (C.c_int, [_vp]),
    "graph_dirty_out_count": (_sz, [_vp]),
    "graph_dirty_in_count": (_sz, [_vp]),
    "graph_compact": (None, [_vp]),
    "graph_maybe_compact": (C.c_int, [_vp, C.c_double]),
    "graph_ensure_vertex": (None, [_vp, C.c_uint32]),
    "graph_base_edge_count_directed": (_sz, [_vp]),
    "graph_compact_neighbors": (_sz, [_vp, C.c_uint32, _u32p, _sz]),
    "graph_compact_in_neighbors": (_sz, [_vp, C.c_uint32, _u32p, _sz]),
    "bfs_create": (_vp, [_vp, C.c_uint32, C.c_double]),
    "bfs_destroy": (None, [_vp]),
    "bfs_recompute": (None, [_vp]),
    "bfs_apply": (C.c_int, [_vp, _u32p, _u32p, _u8p, _sz]),
    "bfs_distances": (_sz, [_vp, _u32p, _sz]),
    "bfs_reachable_count": (_sz, [_vp]),
    "bfs_last_deletion_candidates": (_sz, [_vp]),
    "bfs_last_affected_vertices": (_sz, [_vp]),
    "bfs_last_used_full_recompute": (C.c_int, [_vp]),
}


def build() -> None:
    """Compile the oracle (and the reference shim when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def available(kind: str = "port") -> bool:
    return os.path.exists(_PATHS[kind])


class _Lib:
    def __init__(self, kind: str):
        if not available(kind):
            raise FileNotFoundError(f"oracle library {_PATHS[kind]} is not built")
        self.kind = kind
        self.dll = C.CDLL(_PATHS[kind])
        p = _PREFIX[kind]
        for name, (res, args) in _SIGS.items():
            fn = getattr(self.dll, p + name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)
        if kind == "reference":
            self.dll.vxr_csr_create.restype = _vp
            self.dll.vxr_csr_create.argtypes = [_u32p, _sz, C.c_int]
            self.dll.vxr_csr_destroy.argtypes = [_vp]
            self.dll.vxr_csr_vertex_count.restype = _sz
            self.dll.vxr_csr_vertex_count.argtypes = [_vp]
            self.dll.vxr_csr_multi_bfs.restype = C.c_int
            self.dll.vxr_csr_multi_bfs.argtypes = [_vp, _u32p, _sz, C.c_int, _u64p, _u32p]
        else:
            self.dll.vxo_csr_bfs.restype = C.c_int
            self.dll.vxo_csr_bfs.argtypes = [_u64p, _u32p, _sz, C.c_uint32, _u32p]


def load(kind: str = "port") -> _Lib:
    if kind not in _LIBS:
        _LIBS[kind] = _Lib(kind)
    return _LIBS[kind]


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _batch(src, dst, add):
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    a = np.ascontiguousarray(add, dtype=np.uint8)
    assert s.shape == d.shape == a.shape
    return s, d, a


class OracleGraph:
    """DynamicGraph semantics (include/velographx/storage/dynamic_graph.hpp)."""

    def __init__(self, vertices: int = 0, directed: bool = False, kind: str = "port"):
        self.lib = load(kind)
        self.directed = directed
        self.h = self.lib.graph_create(vertices, int(directed))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.graph_destroy(h)
            self.h = None

    @property
    def vertex_count(self) -> int:
        return self.lib.graph_vertex_count(self.h)

    @property
    def version(self) -> int:
        return self.lib.graph_version(self.h)

    def bulk_load_edges(self, edges) -> None:
        uv = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1, 2))
        self.lib.graph_bulk_load(self.h, _ptr(uv, _u32p), uv.shape[0])

    def apply(self, src, dst, add) -> None:
        s, d, a = _batch(src, dst, add)
        self.lib.graph_apply(self.h, _ptr(s, _u32p), _ptr(d, _u32p), _ptr(a, _u8p), s.size)

    def _row(self, fn, u):
        n = fn(self.h, u, None, 0)
        out = np.zeros(max(n, 1), dtype=np.uint32)
        fn(self.h, u, _ptr(out, _u32p), n)
        return out[:n].tolist()

    def neighbors(self, u: int):
        return self._row(self.lib.graph_neighbors, u)

    def in_neighbors(self, v: int):
        return self._row(self.lib.graph_in_neighbors, v)

    def compact_neighbors(self, u: int):
        return self._row(self.lib.graph_compact_neighbors, u)

    def compact_in_neighbors(self, v: int):
        return self._row(self.lib.graph_compact_in_neighbors, v)

    def ensure_vertex(self, v: int) -> None:
        self.lib.graph_ensure_vertex(self.h, v)

    def base_edge_count_directed(self) -> int:
        return self.lib.graph_base_edge_count_directed(self.h)

    def has_edge(self, u: int, v: int) -> bool:
        return bool(self.lib.graph_has_edge(self.h, u, v))

    def edge_count_directed(self) -> int:
        return self.lib.graph_edge_count_directed(self.h)

    def delta_edge_count(self) -> int:
        return self.lib.graph_delta_edge_count(self.h)

    def is_compact(self) -> bool:
        return bool(self.lib.graph_is_compact(self.h))

    def dirty_out_count(self) -> int:
        return self.lib.graph_dirty_out_count(self.h)

    def dirty_in_count(self) -> int:
        return self.lib.graph_dirty_in_count(self.h)

    def compact(self) -> None:
        self.lib.graph_compact(self.h)

    def maybe_compact(self, threshold: float = 0.25) -> bool:
        return bool(self.lib.graph_maybe_compact(self.h, threshold))

    def csr(self):
        """Logical out-adjacency as (offsets u64[V+1], cols u32[A])."""
        V = self.vertex_count
        rows = [self.neighbors(u) for u in range(V)]
        off = np.zeros(V + 1, dtype=np.uint64)
        off[1:] = np.cumsum([len(r) for r in rows])
        cols = np.array([x for r in rows for x in r], dtype=np.uint32)
        return off, cols


class OracleBFS:
    """BasicIncrementalBFS<DynamicGraph> (include/velographx/incremental/bfs.hpp)."""

    def __init__(self, graph: OracleGraph, source: int, deletion_fallback_fraction: float = 0.35):
        self.graph = graph
        self.lib = graph.lib
        self.h = self.lib.bfs_create(graph.h, source, deletion_fallback_fraction)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.bfs_destroy(h)
            self.h = None

    def apply(self, src, dst, add) -> None:
        s, d, a = _batch(src, dst, add)
        self.lib.bfs_apply(self.h, _ptr(s, _u32p), _ptr(d, _u32p), _ptr(a, _u8p), s.size)

    def recompute(self) -> None:
        self.lib.bfs_recompute(self.h)

    def distances(self) -> np.ndarray:
        n = self.lib.bfs_distances(self.h, None, 0)
        out = np.empty(n, dtype=np.uint32)
        if n:
            self.lib.bfs_distances(self.h, _ptr(out, _u32p), n)
        return out

    @property
    def reachable_count(self) -> int:
        return self.lib.bfs_reachable_count(self.h)

    @property
    def last_deletion_candidates(self) -> int:
        return self.lib.bfs_last_deletion_candidates(self.h)

    @property
    def last_affected_vertices(self) -> int:
        return self.lib.bfs_last_affected_vertices(self.h)

    @property
    def last_used_full_recompute(self) -> bool:
        return bool(self.lib.bfs_last_used_full_recompute(self.h))

    def stats(self):
        return (self.reachable_count, self.last_deletion_candidates,
                self.last_affected_vertices, self.last_used_full_recompute)


def csr_multi_bfs(edges: np.ndarray, roots: np.ndarray, threads: int, directed: bool = False,
                  want_dist: bool = False):
    """The reference's thread-per-root static BFS (reference back end only).

    Returns (V, reached_arcs u64[k], dist u32[k,V] or None)."""
    lib = load("reference")
    uv = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1, 2))
    h = lib.dll.vxr_csr_create(_ptr(uv, _u32p), uv.shape[0], int(directed))
    try:
        V = lib.dll.vxr_csr_vertex_count(h)
        r = np.ascontiguousarray(roots, dtype=np.uint32)
        arcs = np.zeros(r.size, dtype=np.uint64)
        dist = np.empty((r.size, V), dtype=np.uint32) if want_dist else None
        rc = lib.dll.vxr_csr_multi_bfs(h, _ptr(r, _u32p), r.size, threads, _ptr(arcs, _u64p),
                                       _ptr(dist, _u32p) if want_dist else None)
        if rc != 0:
            raise ValueError("reference bfs_distances failed (root out of range)")
        return V, arcs, dist
    finally:
        lib.dll.vxr_csr_destroy(h)
