"""Per-batch replay of an update stream through the CPU reference (test
infrastructure and the benchmark's CPU-baseline leg only).

``replay`` drives ``DynamicGraph`` + ``IncrementalBFS::apply``
(include/velographx/incremental/bfs.hpp:29-98) batch by batch -- the unmodified
reference (``kind="reference"``, oracle/_ref) when it is built, else the C
restatement (``kind="port"``) -- and records after every batch what the GPU
path must reproduce bit for bit: a 64-bit digest of the distance vector, its
length, and the four counters of bfs.hpp:23-27.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from .oracle import OracleBFS, OracleGraph, available


def digest(dist: np.ndarray) -> int:
    """Sum over v of splitmix64((v << 32) | dist[v]) modulo 2^64 (the GPU
    library's vx_bfs_digest)."""
    d = np.ascontiguousarray(dist, dtype=np.uint32).astype(np.uint64)
    v = np.arange(d.size, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (v << np.uint64(32)) | d
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        return int(np.sum(z, dtype=np.uint64))


@dataclass
class BatchRecord:
    digest: int
    length: int
    reachable: int
    candidates: int
    affected: int
    full: bool


def best_kind() -> str:
    return "reference" if available("reference") else "port"


class Replay:
    """The reference's state machine on one graph: bulk load, BFS from root,
    then batches applied one call at a time.  ``apply_timed`` returns the
    seconds of the apply call alone (the digest is taken outside it)."""

    def __init__(self, edges: np.ndarray, vertices: int, root: int, directed: bool = False,
                 fraction: float = 0.35, kind: str | None = None):
        self.kind = kind or best_kind()
        self.g = OracleGraph(vertices, directed, self.kind)
        self.g.bulk_load_edges(edges)
        self.b = OracleBFS(self.g, root, fraction)
        self.fraction = fraction

    def apply_timed(self, src, dst, add) -> float:
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        a = np.ascontiguousarray(add, dtype=np.uint8)
        t0 = time.perf_counter()
        self.b.apply(s, d, a)
        return time.perf_counter() - t0

    def recompute_timed(self) -> float:
        t0 = time.perf_counter()
        self.b.recompute()
        return time.perf_counter() - t0

    def record(self) -> BatchRecord:
        dist = self.b.distances()
        r, c, a, f = self.b.stats()
        return BatchRecord(digest(dist), int(dist.size), int(r), int(c), int(a), bool(f))


def fallback_limit(vertices: int, fraction: float) -> int:
    """max(1, size_t(double(V) * fraction))  (bfs.hpp:225-226)."""
    return max(1, int(float(vertices) * fraction))


def mismatch(gpu: BatchRecord, ref: BatchRecord, pre_vertices: int, fraction: float) -> str | None:
    """None when the GPU's post-batch state equals the reference's; else what
    differs.  On a fallback batch the reference's affected counter is the
    count at which its FIFO walk stopped (an order-dependent value); there the
    GPU's count must also exceed the fallback limit."""
    if gpu.length != ref.length:
        return f"distance length {gpu.length} != {ref.length}"
    if gpu.digest != ref.digest:
        return "distance digest differs"
    if gpu.reachable != ref.reachable:
        return f"reachable {gpu.reachable} != {ref.reachable}"
    if gpu.candidates != ref.candidates:
        return f"deletion candidates {gpu.candidates} != {ref.candidates}"
    if gpu.full != ref.full:
        return f"full-recompute flag {gpu.full} != {ref.full}"
    if ref.full:
        if gpu.affected <= fallback_limit(pre_vertices, fraction):
            return f"fallback with affected {gpu.affected} not above the limit"
    elif gpu.affected != ref.affected:
        return f"affected {gpu.affected} != {ref.affected}"
    return None
