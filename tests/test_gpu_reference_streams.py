"""GPU against the CPU reference after every batch, at the benchmark
configurations' sizes.

Each test replays the same seeded stream through the reference's
``DynamicGraph`` + ``IncrementalBFS::apply`` (oracle/_ref when it is built,
else the pinned C restatement) and through the GPU path, and compares after
every batch the distance vector (64-bit digest and length) and the four
counters of include/velographx/incremental/bfs.hpp:23-27.

* undirected R-MAT scale 22, 10,000-op batches (70% insertions, 30% deletions
  of loaded edges), through the default per-batch ``apply`` and through the
  batched stream path;
* undirected R-MAT scale 20, the first 100 batches of the lognormal stream
  (median 500 ops, sigma 2, 80% insertions), batched and per batch;
* the 4096 x 4096 lattice with 0.1% long-range edges, root at corner 0,
  1,000-op batches with half of them deletions near the root.
"""
import numpy as np
import pytest

import workloads as w
from oracle.replay import BatchRecord, Replay, mismatch

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("velographx_b200")


def gpu_record(g, b) -> BatchRecord:
    st = b.stats()
    return BatchRecord(int(b.digest()), int(g.vertex_count), int(st["reachable_count"]),
                       int(st["last_deletion_candidates"]), int(st["last_affected_vertices"]),
                       bool(st["last_used_full_recompute"]))


def stream_records(digs, stats, V) -> list:
    """Per-batch records of apply_stream(digests=True, stats=True); the stream
    reports the reachable count modulo 2^32 (exact below 2^32 vertices)."""
    return [BatchRecord(int(digs[t]), V, int(stats[t, 3]), int(stats[t, 0]), int(stats[t, 1]), bool(stats[t, 2]))
            for t in range(len(digs))]


def check_all(name, gpu, ref_replay, stream, V, fraction=0.35):
    bad = []
    for t in range(len(gpu)):
        ref_replay.apply_timed(*stream.batch(t))
        ref = ref_replay.record()
        why = mismatch(gpu[t], ref, V, fraction)
        if why:
            bad.append(f"{name} batch {t}: {why}")
    assert not bad, bad[:5]
    return len(gpu)


def test_rmat22_10k_batches_every_batch_equals_reference():
    scale, seed, nb = 22, 22, 20
    V = 1 << scale
    e = w.rmat_edges(scale, 16, seed=seed)
    root = int(w.non_isolated_roots(e, V, 64, seed=seed + 1)[0])
    st = w.mixed_stream(e, V, [10_000] * nb, 0.7, seed=seed + 2)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, root)
    plain = []
    for t in range(nb):
        b.apply_arrays(*st.batch(t))
        plain.append(gpu_record(g, b))
    del b, g
    g2 = vx.Graph(V, False)
    g2.bulk_load_edges(e)
    b2 = vx.IncrementalBFS(g2, root)
    digs, stats = b2.apply_stream(st.src, st.dst, st.add, st.offsets.astype(np.uint64), digests=True, stats=True)
    batched = stream_records(digs, stats, V)
    del b2, g2
    for t in range(nb):
        assert batched[t] == plain[t], f"batched and per-batch paths differ after batch {t}"
    n = check_all("rmat22", plain, Replay(e, V, root), st, V)
    assert n == nb


def test_rmat20_lognormal_first_100_batches_equal_reference():
    scale, seed, nb = 20, 33, 100
    V = 1 << scale
    e = w.rmat_edges(scale, 16, seed=seed)
    root = w.max_degree_root(e, V)
    sizes = w.lognormal_sizes(1000, median=500.0, sigma=2.0, lo=1, hi=200_000, seed=seed + 1)
    st = w.mixed_stream(e, V, sizes, 0.8, seed=seed + 2).prefix(nb)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, root)
    digs, stats = b.apply_stream(st.src, st.dst, st.add, st.offsets.astype(np.uint64), digests=True, stats=True)
    batched = stream_records(digs, stats, V)
    final = b.distances_array()
    del b, g
    g2 = vx.Graph(V, False)
    g2.bulk_load_edges(e)
    b2 = vx.IncrementalBFS(g2, root)
    for t in range(nb):
        b2.apply_arrays(*st.batch(t))
        assert gpu_record(g2, b2) == batched[t], f"per-batch and batched paths differ after batch {t}"
    assert np.array_equal(b2.distances_array(), final)
    del b2, g2
    assert check_all("lognormal", batched, Replay(e, V, root), st, V) == nb


def test_grid4096_near_root_deletions_every_batch_equals_reference():
    side, seed, nb, ops = 4096, 44, 20, 1000
    V = side * side
    e = w.grid_edges(side, side, 0.001, seed=seed)
    g = vx.Graph(V, False)
    g.bulk_load_edges(e)
    b = vx.IncrementalBFS(g, 0)
    # the first nb batches of the benchmark's 500-batch stream
    st = w.near_root_stream(e, V, b.distances_array(), 500, ops, 0.5, seed + 1).prefix(nb)
    recs = []
    for t in range(nb):
        b.apply_arrays(*st.batch(t))
        recs.append(gpu_record(g, b))
    del b, g
    assert check_all("grid4096", recs, Replay(e, V, 0), st, V) == nb
