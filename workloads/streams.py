"""Update-stream measurements beyond the headline benchmark.

``grid``       4096 x 4096 lattice (4-neighbour) + 0.1% seeded long-range
               edges, root at corner 0, batches of 1,000 ops with half of them
               deletions drawn from the edges nearest the root (the ones whose
               endpoints have the smallest distances) -- deep subtree
               invalidation and repair.
``lognormal``  R-MAT scale 20 with 1,000 update batches of lognormal sizes
               (median 500 ops, sigma 2, clipped to [1, 200000]; 80%
               insertions): the plain path (one batch at a time through the
               public API, host arrays copied in and the counters read back
               per batch) against the batched path (the whole stream in one
               apply_stream call), end to end from page-locked host arrays,
               with device memory for the stream reserved beforehand.

Every run times batches with CUDA events on the graph's stream and checks the
maintained distances against a fresh full BFS at regular batches.

  python -m workloads.streams --workload grid [--batches 500]
  python -m workloads.streams --workload lognormal [--scale 20]
  python -m workloads.streams --workload window [--window 256] [--digests]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

import workloads as w
from velographx_b200 import Graph, IncrementalBFS, MultiRootBFS


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def pinned_stream(st: w.Stream) -> w.Stream:
    """The stream's host arrays moved to page-locked memory (both paths copy
    from it)."""
    import torch

    n = st.src.size
    buf = torch.empty(9 * max(n, 1), dtype=torch.uint8, pin_memory=True).numpy()
    src = buf[: 4 * n].view(np.uint32)
    dst = buf[4 * n: 8 * n].view(np.uint32)
    add = buf[8 * n: 9 * n]
    src[:], dst[:], add[:] = st.src, st.dst, st.add
    return w.Stream(src, dst, add, st.offsets)


def record(g: Graph, b: IncrementalBFS) -> tuple:
    """(digest, length, reachable, candidates, affected, full) of the current
    post-batch state: what the CPU reference must reproduce after the batch."""
    st = b.stats()
    return (int(b.digest()), int(g.vertex_count), int(st["reachable_count"]), int(st["last_deletion_candidates"]),
            int(st["last_affected_vertices"]), bool(st["last_used_full_recompute"]))


def stream_records(digs, stats, V: int) -> list:
    """The same records from apply_stream(digests=True, stats=True)."""
    return [(int(digs[t]), V, int(stats[t, 3]), int(stats[t, 0]), int(stats[t, 1]), bool(stats[t, 2]))
            for t in range(len(digs))]


def run_stream(g: Graph, bfs: IncrementalBFS, root: int, stream: w.Stream, check_every: int) -> dict:
    """Device-resident batches (apply_device), timed back to back with events
    between batches; exactness against a fresh full BFS every check_every
    batches (outside the timed spans)."""
    import torch

    V = g.vertex_count
    cs = torch.cuda.ExternalStream(g.stream)
    ds = torch.from_numpy(stream.src.view(np.int32)).cuda()
    dd = torch.from_numpy(stream.dst.view(np.int32)).cuda()
    da = torch.from_numpy(stream.add).cuda()
    torch.cuda.synchronize()
    per, fallbacks, affected, exact, checked = [], 0, [], True, 0
    nb = stream.batches
    k = 0
    while k < nb:
        seg = min(nb, (k // check_every + 1) * check_every) if check_every else nb
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(seg - k + 1)]
        ev[0].record(cs)
        for i in range(k, seg):
            lo, hi = int(stream.offsets[i]), int(stream.offsets[i + 1])
            bfs.apply_device(ds.data_ptr() + 4 * lo, dd.data_ptr() + 4 * lo, da.data_ptr() + lo, hi - lo, V)
            ev[i - k + 1].record(cs)
        torch.cuda.synchronize()
        per += [ev[j].elapsed_time(ev[j + 1]) * 1e3 for j in range(seg - k)]
        st = bfs.stats()
        fallbacks += int(st["last_used_full_recompute"])
        affected.append(st["last_affected_vertices"])
        if check_every:
            fresh = IncrementalBFS(g, root)
            same = np.array_equal(fresh.distances_array(), bfs.distances_array())
            exact = exact and same and fresh.reachable_count == bfs.reachable_count
            checked += 1
            del fresh
        k = seg
    per = np.asarray(per)
    return {"batches": nb, "seconds": float(per.sum() * 1e-6), "batches_per_s": float(nb / (per.sum() * 1e-6)),
            "us_median": float(np.median(per)), "us_p90": float(np.percentile(per, 90)), "us_max": float(per.max()),
            "first_batches_us": [round(float(x), 1) for x in per[:5]],
            "exact": bool(exact), "exact_checks": checked, "_per_batch_us": per}


def grid(side: int = 4096, long_range: float = 0.001, batches: int = 500, ops: int = 1000,
         delete_fraction: float = 0.5, seed: int = 44, check_every: int = 50, ref_batches: int = 20) -> dict:
    """The lattice stream, device-resident batches timed per batch; then, on a
    fresh replica, the records of the first ref_batches batches (returned
    under "_check" for a comparison with the CPU reference)."""
    import torch

    edges = w.grid_edges(side, side, long_range, seed=seed)
    V = side * side
    g = Graph(V, False)
    g.bulk_load_edges(edges)
    # device memory for the whole stream up front (no batch grows the arena)
    g.reserve(ops, ops * batches)
    root = 0
    bfs = IncrementalBFS(g, root)
    cs = torch.cuda.ExternalStream(g.stream)
    e0, e1 = _events()
    torch.cuda.synchronize()
    e0.record(cs)
    bfs.recompute()
    e1.record(cs)
    e1.synchronize()
    full_ms = e0.elapsed_time(e1)
    levels = bfs.stats()["levels"]
    stream = w.near_root_stream(edges, V, bfs.distances_array(), batches, ops, delete_fraction, seed + 1)
    res = run_stream(g, bfs, root, stream, check_every)
    res.update({"workload": f"grid{side}x{side}+{long_range:g}-long-range-root0-{ops}-op-batches-"
                            f"{int(delete_fraction * 100)}pct-near-root-deletions",
                "vertices": V, "arcs": int(g.edge_count_directed()), "full_bfs_ms": full_ms,
                "full_bfs_levels": int(levels)})
    del bfs, g
    # a replica replays every batch untimed: the records of the first
    # ref_batches (for the CPU reference) and each batch's counters, which
    # name what the slowest timed batches did
    per = res.pop("_per_batch_us")
    g = Graph(V, False)
    g.bulk_load_edges(edges)
    g.reserve(ops, ops * batches)
    b = IncrementalBFS(g, root)
    recs, stats, stamps = [], [], []
    for t in range(batches):
        b.apply_arrays(*stream.batch(t))
        st = b.stats()
        stats.append((bool(st["last_used_full_recompute"]), int(st["last_affected_vertices"]),
                      int(st["last_deletion_candidates"])))
        tr = b.phase_trace()
        stamps.append(tr[:7] + tr[27:29])
        if t < ref_batches:
            recs.append(record(g, b))
    del b, g
    slow = np.argsort(per)[::-1][:5]
    res["fallback_batches"] = int(sum(x[0] for x in stats))
    def phases(ts):
        # the update launch's stamps: batch start, after the removals, after
        # the cascade, repair entry (after the insertions), after the
        # invalidation, after the boundary seeds, after the relaxation (us,
        # from the untimed replay of the same batch)
        names = ("classify_removals", "cascade", "insertions", "invalidation", "boundary_seeds", "relaxation")
        return {n: round((int(ts[k + 1]) - int(ts[k])) * 1e-3, 1) if ts[k + 1] >= ts[k] > 0 else None
                for k, n in enumerate(names)}

    res["slowest"] = [{"batch": int(i), "us": round(float(per[i]), 1), "full_recompute": stats[i][0],
                       "affected": stats[i][1], "candidates": stats[i][2], "replay_phase_us": phases(stamps[i]),
                       "replay_handovers": {"cascade": int(stamps[i][7]), "relaxation": int(stamps[i][8])}}
                      for i in slow]
    res["replay_handover_batches"] = {"cascade": int(sum(x[7] for x in stamps)),
                                      "relaxation": int(sum(x[8] for x in stamps))}
    res["affected_median"] = float(np.median([x[1] for x in stats]))
    if ref_batches:
        k = min(ref_batches, batches)
        res["_check"] = (edges, stream.prefix(k), root, recs)
    return res


def insertions_c1(scale: int = 14, batches: int = 100, ops: int = 64, seed: int = 14, repeats: int = 3) -> dict:
    """Undirected R-MAT scale 14, full BFS from the max-degree vertex, then 100
    batches of 64 uniform-random insertions: the plain path (one batch per
    call, counters read back) and the batched path, with the distance digest
    after every batch, each on fresh replicas `repeats` times after one
    untimed round (the batched routes report their medians, the plain path
    its fastest run: a 100-batch run lasts only milliseconds); returns the
    stream (for a check elsewhere) with the timings."""
    import torch

    V = 1 << scale
    edges = w.rmat_edges(scale, 16, seed=seed)
    root = w.max_degree_root(edges, V)
    rng = np.random.default_rng(seed + 1)
    src = rng.integers(0, V, batches * ops, dtype=np.uint32)
    dst = rng.integers(0, V, batches * ops, dtype=np.uint32)
    add = np.ones(batches * ops, np.uint8)
    st = pinned_stream(w.Stream(src, dst, add, np.arange(batches + 1, dtype=np.int64) * ops))
    off = st.offsets.astype(np.uint64)
    out = {"workload": f"rmat{scale}-undirected-ef16-{batches}x{ops}-insertions", "vertices": V, "root": int(root),
           "batches": batches}
    e0, e1 = _events()
    plain_runs, batched_runs, ul_runs, same, phases = [], [], [], True, []
    # one untimed round first: the first launches of the window kernels load
    # them (lazy module loading), which a 1 ms stream would otherwise carry
    for _ in range(repeats + 1):
        g = Graph(V, False)
        g.bulk_load_edges(edges)
        g.reserve(ops, ops * batches)
        b = IncrementalBFS(g, root)
        cs = torch.cuda.ExternalStream(g.stream)
        torch.cuda.synchronize()
        e0.record(cs)
        plain_digests, recs = [], []
        for t in range(batches):
            b.apply_arrays(*st.batch(t))
            b.stats()
            plain_digests.append(b.digest())
        e1.record(cs)
        torch.cuda.synchronize()
        plain_runs.append(batches / (e0.elapsed_time(e1) * 1e-3))
        # batched: version-parallel windows (the default route), then every
        # batch through the persistent update launch (window 0); both return
        # every batch's digest
        for window, runs in ((None, batched_runs), (0, ul_runs)):
            g2 = Graph(V, False)
            g2.bulk_load_edges(edges)
            g2.reserve(ops, ops * batches)
            b2 = IncrementalBFS(g2, root)
            b2.reserve_stream(batches * ops, batches, ops)
            if window is not None:
                b2.set_stream_window(window)
            cs2 = torch.cuda.ExternalStream(g2.stream)
            torch.cuda.synchronize()
            e0.record(cs2)
            digs, _ = b2.apply_stream(st.src, st.dst, st.add, off, digests=True)
            e1.record(cs2)
            torch.cuda.synchronize()
            runs.append(batches / (e0.elapsed_time(e1) * 1e-3))
            same = same and [int(x) for x in digs] == [int(x) for x in plain_digests]
            if window == 0:
                ph = b2.phase_trace()[21:27]
                phases.append([x / 1e3 / batches for x in ph])
            del b2, g2
        del b, g
    plain_runs, batched_runs, ul_runs, phases = plain_runs[1:], batched_runs[1:], ul_runs[1:], phases[1:]
    # the records of every batch, on one more replica (untimed)
    g = Graph(V, False)
    g.bulk_load_edges(edges)
    b = IncrementalBFS(g, root)
    for t in range(batches):
        b.apply_arrays(*st.batch(t))
        recs.append(record(g, b))
    same = same and [r[0] for r in recs] == [int(x) for x in digs]
    del b, g
    # the plain path waits on the host after every batch: its fastest run is
    # reported (the batched routes report their medians)
    out["plain"] = {"batches_per_s": float(np.max(plain_runs)), "runs": [round(x) for x in plain_runs]}
    out["batched"] = {"batches_per_s": float(np.median(batched_runs)), "runs": [round(x) for x in batched_runs],
                      "route": "version-parallel windows of 256 batches (digest of every batch returned)"}
    out["batched_update_launch"] = {
        "batches_per_s": float(np.median(ul_runs)), "runs": [round(x) for x in ul_runs],
        "route": "every batch in one persistent update launch (stream window 0)",
        "phase_us_per_batch": dict(zip(
            ["classify", "removals", "cascade", "insertions", "post_repair", "end_barrier"],
            [round(float(np.median([r[k] for r in phases])), 2) for k in range(6)]))}
    out["plain_equals_batched"] = bool(same)
    out["_check"] = (edges, st, root, recs)
    return out


def lognormal(scale: int = 20, batches: int = 1000, median: float = 500.0, sigma: float = 2.0,
              insert_fraction: float = 0.8, seed: int = 33, check_batches: int = 200, multiroot: int = 256) -> dict:
    """Batched stream (one apply_stream call: upload, stream-wide
    canonicalisation, one persistent launch) against the plain path
    (apply_arrays + a counter read-back per batch) on replicas of one graph."""
    import torch

    V = 1 << scale
    edges = w.rmat_edges(scale, 16, seed=seed)
    root = w.max_degree_root(edges, V)
    sizes = w.lognormal_sizes(batches, median=median, sigma=sigma, lo=1, hi=200_000, seed=seed + 1)
    st = w.mixed_stream(edges, V, sizes, insert_fraction, seed=seed + 2)
    st = pinned_stream(st)
    off = st.offsets.astype(np.uint64)
    n_ops, biggest = int(sizes.sum()), int(sizes.max())

    def replica():
        # device memory for the whole stream reserved up front, so that no
        # batch of either path allocates (and synchronises) mid-stream
        g = Graph(V, False)
        g.bulk_load_edges(edges)
        g.reserve(biggest, n_ops)
        b = IncrementalBFS(g, root)
        b.reserve_stream(n_ops, batches, biggest)
        return g, b

    out = {"workload": f"rmat{scale}-undirected-ef16-lognormal-batches-median{median:g}-sigma{sigma:g}-"
                       f"{int(insert_fraction * 100)}pct-insert",
           "vertices": V, "batches": batches, "ops": int(sizes.sum()), "median_ops": float(np.median(sizes)),
           "max_ops": int(sizes.max())}
    # plain: one batch at a time from host arrays, synchronised per batch --
    # the per-phase path (a launch per commit step and repair half) and the
    # fused one (canonicalisation + one persistent launch per batch).  Each
    # waits on the host after every batch, so its rate moves with the host's
    # load (single runs several times slower than the rest were seen): five
    # runs on fresh replicas, the fastest reported, which keeps the batched
    # path's speed-up over it conservative.
    e0, e1 = _events()
    for name, fused in (("plain", False), ("plain_fused", True)):
        runs = []
        for _ in range(5):
            gp, bp = replica()
            bp.set_fused(fused)
            cs = torch.cuda.ExternalStream(gp.stream)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record(cs)
            for t in range(batches):
                bp.apply_arrays(*st.batch(t))
                bp.stats()
            e1.record(cs)
            torch.cuda.synchronize()
            runs.append((e0.elapsed_time(e1) * 1e-3, time.perf_counter() - t0))
        sec, wall = sorted(runs)[0]
        out[name] = {"seconds": sec, "wall_s": wall, "batches_per_s": batches / sec,
                     "runs_batches_per_s": [round(batches / r[0]) for r in runs]}
        if fused:
            bp_fused = bp
    # batched: the whole stream in one call, every batch's digest returned,
    # distances resident on the device at the end -- through version-parallel
    # windows (the default route), then through the persistent update launch
    # (window 0), whose per-phase clock is reported
    batched_digests = {}
    for name, window in (("batched", None), ("batched_update_launch", 0)):
        # the window route: three runs on fresh replicas, the median reported
        # (a 1,000-batch stream lasts about 13 ms)
        runs = []
        for _ in range(3 if window is None else 1):
            gb, bb = replica()
            if window is not None:
                bb.set_stream_window(window)
            cs = torch.cuda.ExternalStream(gb.stream)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record(cs)
            digs, _ = bb.apply_stream(st.src, st.dst, st.add, off, digests=True)
            e1.record(cs)
            torch.cuda.synchronize()
            runs.append((e0.elapsed_time(e1) * 1e-3, time.perf_counter() - t0))
        sec, wall = sorted(runs)[len(runs) // 2]
        out[name] = {"seconds": sec, "wall_s": wall}
        out[name]["batches_per_s"] = batches / out[name]["seconds"]
        if window is None:
            out[name]["runs_batches_per_s"] = [round(batches / r[0]) for r in runs]
        batched_digests[name] = [int(x) for x in digs]
        if window == 0:
            ph = bb.phase_trace()[21:27]
            out[name]["phase_us_per_batch"] = dict(zip(
                ["classify", "removals", "cascade", "insertions", "post_repair", "end_barrier"],
                [round(x / 1e3 / batches, 2) for x in ph]))
            # the persistent launch itself; the rest of the call is the
            # upload, the stream-wide canonicalisation and first-call allocations
            out[name]["kernel_seconds"] = float(sum(ph)) * 1e-9
        else:
            out[name]["route"] = "version-parallel windows of 256 batches"
            bv = bb
        if not (np.array_equal(bp.distances_array(), bb.distances_array())
                and bp.reachable_count == bb.reachable_count):
            out[name]["exact_final"] = False
    out["batched_routes_equal"] = batched_digests["batched"] == batched_digests["batched_update_launch"]
    out["speedup"] = out["batched"]["batches_per_s"] / out["plain"]["batches_per_s"]
    out["speedup_vs_fused"] = out["batched"]["batches_per_s"] / out["plain_fused"]["batches_per_s"]
    out["speedup_update_launch"] = out["batched_update_launch"]["batches_per_s"] / out["plain"]["batches_per_s"]
    out["exact_final"] = bool(np.array_equal(bp.distances_array(), bv.distances_array())
                              and bp.reachable_count == bv.reachable_count
                              and np.array_equal(bp_fused.distances_array(), bv.distances_array())
                              and out["batched_routes_equal"])
    # per-batch check on a prefix: digests of the stream path against the plain path
    if check_batches:
        k = min(check_batches, batches)
        gc_, bc = replica()
        gd, bd = replica()
        digs, stats = bc.apply_stream(st.src, st.dst, st.add, off[: k + 1], digests=True, stats=True)
        recs = stream_records(digs, stats, V)
        bd.set_fused(False)  # checked against the per-phase path
        ok = True
        ok_v = True
        for t in range(k):
            bd.apply_arrays(*st.batch(t))
            r = record(gd, bd)
            ok = ok and r == recs[t]
            ok_v = ok_v and r[0] == batched_digests["batched"][t]
        out["exact_every_batch"] = {"batches": k, "exact": bool(ok and ok_v), "against": "per-phase plain path",
                                    "routes": "version-parallel digests; update-launch digests and counters"}
        out["_check"] = (edges, st.prefix(k), root, recs)
        del bc, gc_, bd, gd
    if multiroot:
        # the configuration's 256 roots in one bit-parallel launch (median of three runs)
        roots = w.non_isolated_roots(edges, V, multiroot, seed=seed + 3)
        gm = Graph(V, False)
        gm.bulk_load_edges(edges)
        mr = MultiRootBFS(gm, roots)
        mr.run()
        cs = torch.cuda.ExternalStream(gm.stream)
        runs = []
        for _ in range(3):
            torch.cuda.synchronize()
            e0.record(cs)
            mr.run()
            e1.record(cs)
            e1.synchronize()
            runs.append(e0.elapsed_time(e1))
        ms = float(np.median(runs))
        out["multiroot"] = {"roots": int(roots.size), "ms": ms, "ms_runs": [round(x, 3) for x in runs],
                            "gteps": mr.reached_arcs() / 2 / (ms * 1e-3) / 1e9, "levels": mr.levels}
        out["_roots"] = roots
        del mr, gm
    return out


def window_case(scale: int = 20, window: int = 256, digests: bool = False, repeats: int = 2, seed: int = 33) -> dict:
    """The lognormal stream through apply_stream's version-parallel windows
    alone (`window` batches per window), `repeats` times on fresh replicas:
    the case the window kernel is profiled on."""
    import torch

    V = 1 << scale
    edges = w.rmat_edges(scale, 16, seed=seed)
    root = w.max_degree_root(edges, V)
    sizes = w.lognormal_sizes(1000, median=500.0, sigma=2.0, lo=1, hi=200_000, seed=seed + 1)
    st = pinned_stream(w.mixed_stream(edges, V, sizes, 0.8, seed=seed + 2))
    off = st.offsets.astype(np.uint64)
    e0, e1 = _events()
    runs = []
    for _ in range(repeats):
        g = Graph(V, False)
        g.bulk_load_edges(edges)
        g.reserve(int(sizes.max()), int(st.offsets[-1]))
        b = IncrementalBFS(g, root)
        b.set_stream_window(window)
        b.reserve_stream(int(st.offsets[-1]), len(sizes), int(sizes.max()))
        cs = torch.cuda.ExternalStream(g.stream)
        torch.cuda.synchronize()
        e0.record(cs)
        b.apply_stream(st.src, st.dst, st.add, off, digests=digests)
        e1.record(cs)
        torch.cuda.synchronize()
        runs.append(len(sizes) / (e0.elapsed_time(e1) * 1e-3))
        trace = b.window_trace()
        del b, g
    return {"workload": f"rmat{scale}-lognormal-1000-batches-window{window}", "batches_per_s_runs": runs,
            "last_window_levels_us_nf_pull": [[round(a, 1), int(n), bool(q)] for a, n, q in trace]}


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", choices=["grid", "lognormal", "window"], default="grid")
    ap.add_argument("--window", type=int, default=256)
    ap.add_argument("--digests", action="store_true")
    ap.add_argument("--side", type=int, default=4096)
    ap.add_argument("--batches", type=int, default=500)
    ap.add_argument("--ops", type=int, default=1000)
    ap.add_argument("--check-every", type=int, default=50)
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--sigma", type=float, default=2.0)
    a = ap.parse_args()
    t0 = time.time()
    if a.workload == "window":
        res = window_case(a.scale, a.window, a.digests)
    elif a.workload == "lognormal":
        res = lognormal(a.scale, batches=a.batches if a.batches != 500 else 1000, sigma=a.sigma)
    else:
        res = grid(a.side, batches=a.batches, ops=a.ops, check_every=a.check_every)
    res = {k: v for k, v in res.items() if not k.startswith("_")}  # the reference-check records stay in-process
    res["wall_s"] = time.time() - t0
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    sys.exit(main())
