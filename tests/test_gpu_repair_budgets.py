"""GPU: the time budget of the incremental repair's phases.

On a deep graph one batch can move the distances of a large part of the graph,
and the cascade or the relaxation then walks them level by level.  A phase that
has run longer than a multiple of the last full BFS's time (set_handover, 1 by
default) hands over to a BFS:

- the post-batch relaxation (an inserted shortcut lowers half a lattice): the
  rest of its queue is dropped and a full BFS of the post-batch graph gives the
  distances and the reachable count;
- the deletion cascade (a wall of deleted edges near the root raises a third of
  a lattice): a BFS of the graph without the batch's deletions gives the
  affected set (the vertices whose distance it raises), their count, and the
  fallback decision; the post-batch repair then only relaxes the insertions.

Either way the batch's distances and counters are the ones the reference's
IncrementalBFS::apply reports, checked batch by batch on both the fused and the
per-phase path with the handover at once (multiple 0: at a phase's first
work-ring round), never (negative) and by default.  Entries 27 and 28 of the
phase trace count the batches whose cascade and whose relaxation handed over.
"""
import numpy as np
import pytest

from oracle import OracleBFS, OracleGraph
from tests.helpers import splitmix_digest as digest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import velographx_b200 as vx  # noqa: E402
import workloads as w  # noqa: E402

CASCADE, RELAX = 27, 28  # phase-trace entries of the handover counts


def lattice_batches(side):
    """Batches on a side x side lattice rooted at corner 0: a shortcut from
    the root to the far corner (lowers about half the lattice), its removal
    (raises them again), a shortcut to the middle together with deletions
    near the root, and a quiet batch."""
    far, mid = side * side - 1, (side // 2) * side + side // 2
    return [
        (np.array([0], np.uint32), np.array([far], np.uint32), np.array([1], np.uint8)),
        (np.array([0], np.uint32), np.array([far], np.uint32), np.array([0], np.uint8)),
        (np.array([0, 0, 1, side], np.uint32), np.array([mid, 1, 2, 2 * side], np.uint32),
         np.array([1, 0, 0, 0], np.uint8)),
        (np.array([5], np.uint32), np.array([6], np.uint32), np.array([0], np.uint8)),
    ]


def wall(side, cols, add=()):
    """Deletes the edges between rows 0 and 1 in columns [0, cols): every
    vertex below the wall in those columns loses all its shortest paths
    ((side - 1) * cols affected vertices); add lists extra insertions."""
    s = [np.arange(cols, dtype=np.uint32)]
    d = [np.arange(cols, dtype=np.uint32) + side]
    a = [np.zeros(cols, np.uint8)]
    for u, v in add:
        s.append(np.array([u], np.uint32))
        d.append(np.array([v], np.uint32))
        a.append(np.array([1], np.uint8))
    return np.concatenate(s), np.concatenate(d), np.concatenate(a)


def restore_wall(side, cols):
    return (np.arange(cols, dtype=np.uint32), np.arange(cols, dtype=np.uint32) + side,
            np.ones(cols, np.uint8))


def cascade_batches(side):
    far = side * side - 1
    unlink = (np.array([0], np.uint32), np.array([far], np.uint32), np.array([0], np.uint8))
    return [
        wall(side, 150),                    # 76,650 affected (29%)
        restore_wall(side, 150),            # insertions only
        wall(side, 150, add=[(0, far)]),    # the same wall and a shortcut in one batch
        tuple(np.concatenate(x) for x in zip(restore_wall(side, 150), unlink)),  # the shortcut's region: falls back
        wall(side, 200),                    # 102,200 affected (39%): falls back
        restore_wall(side, 200),
        wall(side, 3),                      # 1,533 affected
        (np.array([9], np.uint32), np.array([10], np.uint32), np.array([0], np.uint8)),
    ]


def run_against_reference(side, batches, fused, handover, expect=None):
    """Applies batches to the device and the reference, comparing distances
    and counters after each; expect[t] = (cascade, relax) handovers of batch t
    (None: not checked)."""
    V = side * side
    edges = w.grid_edges(side, side, 0.0, seed=3)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, 0)
    b.set_fused(fused)
    b.set_handover(handover)
    og = OracleGraph(V, False)
    og.bulk_load_edges(edges)
    ob = OracleBFS(og, 0)
    for t, (s, d, a) in enumerate(batches):
        b.apply_arrays(s, d, a)
        ob.apply(s, d, a)
        assert np.array_equal(b.distances_array(), ob.distances()), t
        st = b.stats()
        r, c, af, full = ob.stats()
        assert st["reachable_count"] == r, t
        assert st["last_deletion_candidates"] == c, t
        assert st["last_used_full_recompute"] == bool(full), t
        if not full:
            assert st["last_affected_vertices"] == af, t
        tr = b.phase_trace()
        if handover < 0:
            assert (tr[CASCADE], tr[RELAX]) == (0, 0), (t, tr[CASCADE:])
        elif expect is not None and expect[t] is not None:
            want_c, want_r = expect[t]
            assert tr[CASCADE] == want_c, (t, tr[CASCADE:])
            if want_r is not None:
                assert tr[RELAX] == want_r, (t, tr[CASCADE:])


@pytest.mark.parametrize("handover", [0.0, -1.0, 1.0])
@pytest.mark.parametrize("fused", [True, False])
def test_relaxation_handover_matches_the_reference(fused, handover):
    side = 256
    quiet = (np.array([7], np.uint32), np.array([8], np.uint32), np.array([0], np.uint8))
    # at multiple 0 the shortcut's relaxation and its removal's cascade hand
    # over; later batches run from a clean repair workspace
    expect = [(0, 1), (1, 0), None, None, None] if handover == 0 else None
    run_against_reference(side, lattice_batches(side) + [quiet], fused, handover, expect)


@pytest.mark.parametrize("handover", [0.0, -1.0, 1.0])
@pytest.mark.parametrize("fused", [True, False])
def test_cascade_handover_matches_the_reference(fused, handover):
    side = 512  # V = 262,144: the fallback above 91,750 affected
    # at multiple 0 every cascade and relaxation that drains its work ring hands over
    expect = [(1, 0), (0, 1), (1, 1), (1, 0), (1, 0), (0, 1), (1, 0), (1, 0)] if handover == 0 else None
    run_against_reference(side, cascade_batches(side), fused, handover, expect)


@pytest.mark.parametrize("handover", [0.0, 1.0])
def test_handovers_inside_one_update_launch_match_the_reference(handover):
    """The same batches as one stream through the persistent update launch
    (apply_stream with per-batch counters): every handover's scratch state is
    back to zero for the next batch of the same launch."""
    side = 512
    V = side * side
    batches = cascade_batches(side)
    src = np.concatenate([b[0] for b in batches])
    dst = np.concatenate([b[1] for b in batches])
    add = np.concatenate([b[2] for b in batches])
    off = np.concatenate([[0], np.cumsum([len(b[0]) for b in batches])]).astype(np.uint64)
    edges = w.grid_edges(side, side, 0.0, seed=3)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    b = vx.IncrementalBFS(g, 0)
    b.set_handover(handover)
    digs, stats = b.apply_stream(src, dst, add, off, digests=True, stats=True)
    if handover == 0:
        assert b.phase_trace()[CASCADE] >= 5  # the wall batches' cascades handed over inside the launch
    og = OracleGraph(V, False)
    og.bulk_load_edges(edges)
    ob = OracleBFS(og, 0)
    for t, (s, d, a) in enumerate(batches):
        ob.apply(s, d, a)
        assert int(digs[t]) == digest(ob.distances()), t
        r, c, af, full = ob.stats()
        assert stats[t, 0] == c and bool(stats[t, 2]) == bool(full) and stats[t, 3] == r, (t, stats[t])
        if not full:
            assert stats[t, 1] == af, t
    assert np.array_equal(b.distances_array(), ob.distances())
