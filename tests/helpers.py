"""Shared helpers for the parity tests."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(d) -> str:
    return hashlib.sha256(np.ascontiguousarray(d, dtype="<u4").tobytes()).hexdigest()


def golden_names():
    return sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json"))


def load_golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def fallback_limit(vertices: int, fraction: float) -> int:
    """max(1, size_t(double(V) * fraction))  (include/velographx/incremental/bfs.hpp:225-226)."""
    return max(1, int(float(vertices) * fraction))


def check_record(rec: dict, dist: np.ndarray, stats, edge_count, version, vertex_count, ctx: str,
                 prev_vertex_count: int, fraction: float) -> None:
    """Compare one post-batch state with a golden record (bit-exact distances).

    stats = (reachable, candidates, affected, full).  When the reference fell back to a
    full recompute, its affected counter is the count at which its FIFO walk stopped (an
    order-dependent value); we then require only that our count also exceeds the limit."""
    assert dist.size == rec["len"], f"{ctx}: distance length {dist.size} != {rec['len']}"
    if "dist" in rec:
        exp = np.asarray(rec["dist"], dtype=np.uint64)
        if not np.array_equal(dist.astype(np.uint64), exp):
            bad = np.flatnonzero(dist.astype(np.uint64) != exp)[:5]
            raise AssertionError(f"{ctx}: distances differ at {bad.tolist()}: got {dist[bad].tolist()} "
                                 f"expected {exp[bad].tolist()}")
    assert digest(dist) == rec["sha256"], f"{ctx}: distance digest differs"
    r, c, a, full = rec["stats"]
    assert stats[0] == r, f"{ctx}: reachable {stats[0]} != {r}"
    assert stats[1] == c, f"{ctx}: deletion candidates {stats[1]} != {c}"
    assert bool(stats[3]) == bool(full), f"{ctx}: full-recompute flag {stats[3]} != {full}"
    if full:
        assert stats[2] > fallback_limit(prev_vertex_count, fraction), f"{ctx}: fallback without exceeding limit"
    else:
        assert stats[2] == a, f"{ctx}: affected {stats[2]} != {a}"
    if edge_count is not None:
        assert edge_count == rec["edge_count"], f"{ctx}: edge count {edge_count} != {rec['edge_count']}"
    assert version == rec["version"], f"{ctx}: version {version} != {rec['version']}"
    assert vertex_count == rec["vertex_count"], f"{ctx}: vertex count {vertex_count} != {rec['vertex_count']}"


def mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def splitmix_digest(dist: np.ndarray) -> int:
    """The library's distance digest: sum over v of mix64(v << 32 | dist[v]) mod 2^64."""
    v = np.arange(dist.size, dtype=np.uint64)
    h = mix64((v << np.uint64(32)) | dist.astype(np.uint64))
    with np.errstate(over="ignore"):
        return int(np.sum(h, dtype=np.uint64))


def messy_stream(edges, V, sizes, seed, grow=0):
    """workloads.mixed_stream (60% insertions) plus duplicates with mixed ops,
    self-loops and (optionally) ids past V."""
    import workloads as w

    rng = np.random.default_rng(seed)
    st = w.mixed_stream(edges, V, sizes, 0.6, seed=seed)
    src, dst, add = st.src.copy(), st.dst.copy(), st.add.copy()
    n = src.size
    if n:
        k = max(1, n // 20)
        i = rng.integers(0, n, k)
        j = rng.integers(0, n, k)
        src[i], dst[i] = src[j], dst[j]  # repeated arcs, mixed ops
        add[i] = rng.integers(0, 2, k).astype(np.uint8)
        loops = rng.integers(0, n, max(1, n // 50))
        dst[loops] = src[loops]
        if grow:
            g_ = rng.integers(0, n, max(1, n // 100))
            dst[g_] = rng.integers(V, V + grow, g_.size).astype(np.uint32)
    return src, dst, add, st.offsets.astype(np.uint64)
