"""Seeded scenarios shared by the golden-vector generator and the tests.

Each scenario is a dict: vertices, directed, edges (N x 2 uint32, bulk
loaded), source, fraction (deletion_fallback_fraction) and batches (a list of
(src, dst, add) uint32/uint32/uint8 arrays).  Inputs depend on numpy only, so
the fixtures do not depend on any product code.
"""
from __future__ import annotations

import hashlib

import numpy as np


def _b(ops):
    """[(u, v, add), ...] -> (src, dst, add) arrays."""
    if not ops:
        return (np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint8))
    a = np.asarray(ops, dtype=np.int64)
    return (a[:, 0].astype(np.uint32), a[:, 1].astype(np.uint32), a[:, 2].astype(np.uint8))


def _sc(vertices, directed, edges, source, fraction, batches):
    e = np.asarray(edges, dtype=np.uint32).reshape(-1, 2)
    return {"vertices": int(vertices), "directed": bool(directed), "edges": e, "source": int(source),
            "fraction": float(fraction), "batches": batches}


def micro() -> dict:
    """The reference's deterministic microcases (tests/test_incremental_bfs_deletion.cpp:57-169,
    tests/test_incremental.cpp:20-31) plus vertex-growth edge cases."""
    diamond = [(0, 1), (0, 2), (1, 3), (2, 3), (3, 4)]
    path20 = [(i, i + 1) for i in range(19)]
    return {
        "micro_alternate_parent": _sc(5, True, diamond, 0, 0.75, [_b([(1, 3, 0)])]),
        "micro_support_fixpoint": _sc(5, True, diamond, 0, 0.90, [_b([(0, 1, 0), (0, 2, 0)])]),
        "micro_surviving_branch": _sc(7, True, [(0, 1), (1, 2), (2, 3), (3, 4), (0, 5), (5, 6), (6, 3)], 0, 0.75,
                                      [_b([(1, 2, 0)])]),
        "micro_mixed": _sc(6, True, [(0, 1), (1, 2), (2, 3), (3, 4), (0, 5)], 0, 0.75, [_b([(1, 2, 0), (5, 3, 1)])]),
        "micro_undirected": _sc(5, False, [(0, 1), (1, 2), (2, 3), (0, 4), (4, 3)], 0, 0.75, [_b([(1, 2, 0)])]),
        "micro_final_state": _sc(5, True, [(0, 1), (1, 2), (2, 3), (3, 4)], 0, 0.75, [_b([(0, 3, 1), (0, 3, 0)])]),
        "micro_fallback": _sc(20, True, path20, 0, 0.05, [_b([(0, 1, 0)])]),
        "micro_out_of_range_source": _sc(4, True, [(0, 1), (1, 2)], 7, 0.75, [_b([(2, 3, 1)])]),
        "micro_path_growth": _sc(5, False, [(0, 1), (1, 2)], 0, 0.35, [_b([(2, 3, 1)])]),
        "micro_growth_and_noops": _sc(3, False, [(0, 1)], 0, 0.35, [
            _b([(1, 2, 1), (2, 2, 1), (7, 7, 0), (5, 9, 0), (1, 2, 1), (2, 6, 1)]),  # self-loops, absent removal, growth
            _b([(6, 2, 0), (2, 6, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0)]),              # last op wins per edge
            _b([(9, 5, 1), (5, 0, 1), (2, 1, 0)]),
        ]),
        "micro_source_grows_later": _sc(3, True, [(0, 1)], 5, 0.35, [_b([(4, 5, 1), (5, 6, 1)])]),
    }


def random_directed(seed=20260830, n=48, m=180, epochs=250, ops=6, fraction=0.75) -> dict:
    """Randomised directed stream shaped like tests/test_incremental_bfs_deletion.cpp:171-210."""
    rng = np.random.default_rng(seed)
    live = set()
    while len(live) < m:
        u, v = (int(x) for x in rng.integers(0, n, 2))
        if u != v:
            live.add((u, v))
    init = sorted(live)
    batches = []
    for _ in range(epochs):
        b = []
        for _ in range(ops):
            if not live or rng.integers(0, 2) == 0:
                for _ in range(30):
                    u, v = (int(x) for x in rng.integers(0, n, 2))
                    if u == v or (u, v) in live:
                        continue
                    live.add((u, v))
                    b.append((u, v, 1))
                    break
            else:
                lst = sorted(live)
                u, v = lst[int(rng.integers(0, len(lst)))]
                live.discard((u, v))
                b.append((u, v, 0))
        batches.append(_b(b))
    return _sc(n, True, init, 0, fraction, batches)


def random_undirected(seed, n=40, steps=400, p_add=0.58) -> dict:
    """Single-op batches on a 40-vertex undirected graph (tests/test_randomized_dynamic.cpp:140-191)."""
    rng = np.random.default_rng(seed)
    batches = []
    for _ in range(steps):
        u, v = (int(x) for x in rng.integers(0, n, 2))
        batches.append(_b([(u, v, int(rng.random() < p_add))]))
    return _sc(n, False, np.zeros((0, 2), np.uint32), 0, 0.35, batches)


def rmat_numpy(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = edge_factor << scale
    u = np.zeros(n, np.uint32)
    v = np.zeros(n, np.uint32)
    for _ in range(scale):
        r = rng.random(n)
        bu = r >= a + b
        bv = ((r >= a) & (r < a + b)) | (r >= a + b + c)
        u = (u << 1) | bu.astype(np.uint32)
        v = (v << 1) | bv.astype(np.uint32)
    return np.stack([u, v], axis=1)


def max_degree_vertex(edges, vertices) -> int:
    e = edges[edges[:, 0] != edges[:, 1]].astype(np.int64)
    key = np.unique(np.minimum(e[:, 0], e[:, 1]) << 32 | np.maximum(e[:, 0], e[:, 1]))
    deg = np.bincount(key >> 32, minlength=vertices) + np.bincount(key & 0xFFFFFFFF, minlength=vertices)
    return int(np.argmax(deg))


def mixed_batches(edges, vertices, batches, size, insert_fraction, seed, near=None) -> list:
    rng = np.random.default_rng(seed)
    simple = edges[edges[:, 0] != edges[:, 1]]
    out = []
    for _ in range(batches):
        add = rng.random(size) < insert_fraction
        src = rng.integers(0, vertices, size=size).astype(np.uint32)
        dst = rng.integers(0, vertices, size=size).astype(np.uint32)
        pool = simple if near is None else near
        pick = rng.integers(0, pool.shape[0], size=size)
        src[~add] = pool[pick[~add], 0]
        dst[~add] = pool[pick[~add], 1]
        out.append((src, dst, add.astype(np.uint8)))
    return out


def rmat14_c1() -> dict:
    """Configuration 1: undirected R-MAT scale 14, root = max-degree vertex, 100 batches of
    64 uniform-random insertions."""
    V = 1 << 14
    e = rmat_numpy(14, seed=14)
    rng = np.random.default_rng(1401)
    batches = [(rng.integers(0, V, 64).astype(np.uint32), rng.integers(0, V, 64).astype(np.uint32),
                np.ones(64, np.uint8)) for _ in range(100)]
    return _sc(V, False, e, max_degree_vertex(e, V), 0.35, batches)


def rmat14_mixed() -> dict:
    V = 1 << 14
    e = rmat_numpy(14, seed=15)
    return _sc(V, False, e, max_degree_vertex(e, V), 0.35, mixed_batches(e, V, 40, 512, 0.7, 1501))


def rmat12_directed() -> dict:
    V = 1 << 12
    e = rmat_numpy(12, seed=12)
    return _sc(V, True, e, max_degree_vertex(e, V), 0.35, mixed_batches(e, V, 40, 256, 0.6, 1201))


def grid_near_root() -> dict:
    """64x64 lattice + 0.1% long-range edges; half of each batch deletes lattice
    edges near the corner root (stresses subtree invalidation)."""
    R = C = 64
    V = R * C
    ed = [(r * C + c, r * C + c + 1) for r in range(R) for c in range(C - 1)]
    ed += [(r * C + c, (r + 1) * C + c) for r in range(R - 1) for c in range(C)]
    lat = np.asarray(ed, np.uint32)
    rng = np.random.default_rng(64)
    extra = rng.integers(0, V, size=(max(1, round(lat.shape[0] * 0.001)), 2)).astype(np.uint32)
    e = np.concatenate([lat, extra])
    near = lat[(lat[:, 0] // C + lat[:, 0] % C) < 12]
    return _sc(V, False, e, 0, 0.35, mixed_batches(e, V, 40, 100, 0.5, 6401, near=near))


def all_scenarios() -> dict:
    s = dict(micro())
    s["random_directed_48"] = random_directed()
    for k in range(3):
        s[f"random_undirected_40_s{k}"] = random_undirected(7919 * (k + 1))
    s["rmat14_c1"] = rmat14_c1()
    s["rmat14_mixed"] = rmat14_mixed()
    s["rmat12_directed"] = rmat12_directed()
    s["grid64_near_root"] = grid_near_root()
    return s


def inputs_digest(sc: dict) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(sc["edges"], dtype="<u4").tobytes())
    for s, d, a in sc["batches"]:
        h.update(np.ascontiguousarray(s, "<u4").tobytes())
        h.update(np.ascontiguousarray(d, "<u4").tobytes())
        h.update(np.ascontiguousarray(a, "u1").tobytes())
    return h.hexdigest()
