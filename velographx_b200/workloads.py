"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Graphs come from the library's host generators (include/vx_workloads.h);
update streams are drawn with numpy's PCG64 from a recorded seed.  The same
arrays feed the GPU path and the CPU oracle.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi

_u32p = C.POINTER(C.c_uint32)


def _lib():
    lib = capi()
    lib.vx_gen_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, _u32p]
    lib.vx_gen_uniform.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, _u32p]
    lib.vx_gen_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, _u32p]
    lib.vx_gen_grid_edge_count.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64]
    lib.vx_gen_grid_edge_count.restype = C.c_uint64
    return lib


def rmat_edges(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
               seed: int = 1) -> np.ndarray:
    """(edge_factor << scale, 2) uint32 R-MAT pairs (self-loops/duplicates kept)."""
    n = edge_factor << scale
    out = np.empty((n, 2), dtype=np.uint32)
    rc = _lib().vx_gen_rmat(scale, edge_factor, a, b, c, seed, out.ctypes.data_as(_u32p))
    if rc != 0:
        raise ValueError("invalid R-MAT parameters")
    return out


def uniform_edges(vertices: int, n: int, seed: int = 1) -> np.ndarray:
    out = np.empty((n, 2), dtype=np.uint32)
    if n:
        _lib().vx_gen_uniform(vertices, n, seed, out.ctypes.data_as(_u32p))
    return out


def grid_edges(rows: int, cols: int, long_range_fraction: float = 0.001, seed: int = 1) -> np.ndarray:
    """4-neighbour lattice plus round(fraction * lattice edges) random long-range edges."""
    lattice = rows * (cols - 1) + (rows - 1) * cols
    extra = int(round(lattice * long_range_fraction))
    lib = _lib()
    n = lib.vx_gen_grid_edge_count(rows, cols, extra)
    out = np.empty((n, 2), dtype=np.uint32)
    lib.vx_gen_grid(rows, cols, extra, seed, out.ctypes.data_as(_u32p))
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


def lognormal_sizes(batches: int, median: float = 500.0, sigma: float = 2.0, lo: int = 1, hi: int = 200_000,
                    seed: int = 11) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = np.exp(np.log(median) + sigma * rng.standard_normal(batches))
    return np.clip(np.rint(s), lo, hi).astype(np.int64)
