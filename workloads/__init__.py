"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Graphs come from ``libvxgen.so`` (``workloads/gen.c``); update streams are
drawn with numpy's PCG64 from a recorded seed.  The same arrays feed the GPU
path and the CPU reference.  This package loads no part of the GPU library,
so the benchmark's reference arm can use it without touching the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvxgen.so")
_u32p = C.POINTER(C.c_uint32)
_LIB = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        lib.vxg_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, _u32p]
        lib.vxg_uniform.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, _u32p]
        lib.vxg_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, _u32p]
        lib.vxg_grid_edge_count.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
        lib.vxg_grid_edge_count.restype = C.c_uint64
        _LIB = lib
    return _LIB


def rmat_edges(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
               seed: int = 1) -> np.ndarray:
    """(edge_factor << scale, 2) uint32 R-MAT pairs (self-loops/duplicates kept)."""
    n = edge_factor << scale
    out = np.empty((n, 2), dtype=np.uint32)
    rc = _lib().vxg_rmat(scale, edge_factor, a, b, c, seed, out.ctypes.data_as(_u32p))
    if rc != 0:
        raise ValueError("invalid R-MAT parameters")
    return out


def uniform_edges(vertices: int, n: int, seed: int = 1) -> np.ndarray:
    out = np.empty((n, 2), dtype=np.uint32)
    if n:
        _lib().vxg_uniform(vertices, n, seed, out.ctypes.data_as(_u32p))
    return out


def grid_edges(rows: int, cols: int, long_range_fraction: float = 0.001, seed: int = 1) -> np.ndarray:
    """4-neighbour lattice plus round(fraction * lattice edges) random long-range edges."""
    lattice = rows * (cols - 1) + (rows - 1) * cols
    extra = int(round(lattice * long_range_fraction))
    lib = _lib()
    n = lib.vxg_grid_edge_count(rows, cols, extra)
    out = np.empty((n, 2), dtype=np.uint32)
    if lib.vxg_grid(rows, cols, extra, seed, out.ctypes.data_as(_u32p)) != 0:
        raise ValueError("invalid lattice size")
    return out


def max_degree_root(edges: np.ndarray, vertices: int) -> int:
    """Highest-degree vertex of the undirected simple graph, ties to the smallest id."""
    e = edges[edges[:, 0] != edges[:, 1]]
    key = np.unique(np.minimum(e[:, 0], e[:, 1]).astype(np.uint64) << 32 | np.maximum(e[:, 0], e[:, 1]))
    u = (key >> 32).astype(np.int64)
    v = (key & 0xFFFFFFFF).astype(np.int64)
    deg = np.bincount(u, minlength=vertices) + np.bincount(v, minlength=vertices)
    return int(np.argmax(deg))


def non_isolated_roots(edges: np.ndarray, vertices: int, k: int, seed: int = 1) -> np.ndarray:
    e = edges[edges[:, 0] != edges[:, 1]]
    present = np.zeros(vertices, dtype=bool)
    present[e[:, 0]] = True
    present[e[:, 1]] = True
    cand = np.flatnonzero(present)
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(cand, size=min(k, cand.size), replace=False)).astype(np.uint32)


@dataclass
class Stream:
    """An update stream: batch b is ops[offsets[b]:offsets[b+1]]."""

    src: np.ndarray
    dst: np.ndarray
    add: np.ndarray
    offsets: np.ndarray

    @property
    def batches(self) -> int:
        return len(self.offsets) - 1

    def batch(self, b: int):
        lo, hi = int(self.offsets[b]), int(self.offsets[b + 1])
        return self.src[lo:hi], self.dst[lo:hi], self.add[lo:hi]

    def prefix(self, k: int) -> "Stream":
        """The first k batches."""
        end = int(self.offsets[k])
        return Stream(self.src[:end], self.dst[:end], self.add[:end], self.offsets[: k + 1])


def mixed_stream(edges: np.ndarray, vertices: int, sizes, insert_fraction: float, seed: int = 7) -> Stream:
    """Batches of uniform-random insertions and deletions of edges sampled from
    the loaded edge list (a deletion of an edge already deleted is a no-op)."""
    rng = np.random.default_rng(seed)
    sizes = np.asarray(sizes, dtype=np.int64)
    total = int(sizes.sum())
    is_add = rng.random(total) < insert_fraction
    src = rng.integers(0, vertices, size=total, dtype=np.uint32)
    dst = rng.integers(0, vertices, size=total, dtype=np.uint32)
    simple = edges[edges[:, 0] != edges[:, 1]]
    pick = rng.integers(0, simple.shape[0], size=total)
    dele = ~is_add
    src[dele] = simple[pick[dele], 0]
    dst[dele] = simple[pick[dele], 1]
    offsets = np.zeros(len(sizes) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    return Stream(src, dst, is_add.astype(np.uint8), offsets)


def insertion_stream(vertices: int, batches: int, ops: int, seed: int) -> Stream:
    """`batches` batches of `ops` uniform-random insertions."""
    rng = np.random.default_rng(seed)
    src = rng.integers(0, vertices, batches * ops, dtype=np.uint32)
    dst = rng.integers(0, vertices, batches * ops, dtype=np.uint32)
    add = np.ones(batches * ops, np.uint8)
    return Stream(src, dst, add, np.arange(batches + 1, dtype=np.int64) * ops)


def near_root_stream(edges: np.ndarray, vertices: int, dist: np.ndarray, batches: int, ops: int,
                     delete_fraction: float, seed: int) -> Stream:
    """Batches of `ops` updates: round(ops * delete_fraction) deletions of edges
    drawn at random from the 2x-sized pool of edges nearest the root (by the
    larger endpoint distance), the rest uniform-random insertions; each batch
    shuffled."""
    rng = np.random.default_rng(seed)
    e = edges[edges[:, 0] != edges[:, 1]]
    nd = int(round(ops * delete_fraction))
    total = nd * batches
    key = np.maximum(dist[e[:, 0]].astype(np.uint64), dist[e[:, 1]].astype(np.uint64))
    pool = np.argsort(key, kind="stable")[: min(e.shape[0], 2 * total)]
    pick = rng.choice(pool, size=total, replace=total > pool.size)
    ni = ops - nd
    src = np.empty(batches * ops, np.uint32)
    dst = np.empty(batches * ops, np.uint32)
    add = np.empty(batches * ops, np.uint8)
    for b in range(batches):
        s = np.concatenate([e[pick[b * nd:(b + 1) * nd], 0], rng.integers(0, vertices, ni, dtype=np.uint32)])
        d = np.concatenate([e[pick[b * nd:(b + 1) * nd], 1], rng.integers(0, vertices, ni, dtype=np.uint32)])
        a = np.concatenate([np.zeros(nd, np.uint8), np.ones(ni, np.uint8)])
        perm = rng.permutation(ops)
        lo = b * ops
        src[lo:lo + ops], dst[lo:lo + ops], add[lo:lo + ops] = s[perm], d[perm], a[perm]
    offsets = np.arange(batches + 1, dtype=np.int64) * ops
    return Stream(src, dst, add, offsets)


def lognormal_sizes(batches: int, median: float = 500.0, sigma: float = 2.0, lo: int = 1, hi: int = 200_000,
                    seed: int = 11) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = np.exp(np.log(median) + sigma * rng.standard_normal(batches))
    return np.clip(np.rint(s), lo, hi).astype(np.int64)


def bfs_levels(edges: np.ndarray, vertices: int, root: int) -> np.ndarray:
    """Unweighted distances from root over the undirected simple graph
    (scipy's breadth-first order; unreachable = 0xFFFFFFFF).  Used to draw
    near-root deletions without the GPU library."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import breadth_first_order

    e = edges[edges[:, 0] != edges[:, 1]]
    m = sp.coo_matrix((np.ones(e.shape[0], np.int8), (e[:, 0], e[:, 1])), shape=(vertices, vertices)).tocsr()
    m = (m + m.T).tocsr()
    order, pred = breadth_first_order(m, root, directed=False, return_predecessors=True)
    dist = np.full(vertices, 0xFFFFFFFF, dtype=np.uint32)
    dist[root] = 0
    for v in order[1:]:
        dist[v] = dist[pred[v]] + 1
    return dist


def digest(dist: np.ndarray) -> int:
    """Order-independent 64-bit digest of a distance vector: the sum over v of
    splitmix64((v << 32) | dist[v]) modulo 2^64 (the library's vx_bfs_digest)."""
    d = np.ascontiguousarray(dist, dtype=np.uint32).astype(np.uint64)
    v = np.arange(d.size, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (v << np.uint64(32)) | d
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        return int(np.sum(z, dtype=np.uint64))
