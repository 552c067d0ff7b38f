#!/usr/bin/env python
"""Benchmark of the B200 dynamic-BFS path (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): undirected
R-MAT scale 22 (4,194,304 vertices, edge factor 16, a=0.57 b=0.19 c=0.19,
seeded, self-loops and duplicates removed), IncrementalBFS from a seeded
non-isolated root, update batches of 10,000 ops (70% uniform-random
insertions, 30% deletions of loaded edges).  One step = one update batch:
Graph.apply + IncrementalBFS repair (device-resident batch for `value`; host
batch through the public API with the counters read back for `e2e`).
Besides the headline, the run reports direction-optimising full BFS from 64
roots (GTEPS and the HBM roofline of the BFS kernel), multi-root BFS of 64
and 256 roots, per-batch exactness against a fresh full BFS, the reference's
CPU path on the host cores, and (under "streams") two further update
streams measured end to end: R-MAT scale 20 with 1,000 lognormal-sized
batches (the batched stream path against the plain one-batch-at-a-time
path) and a 4096 x 4096 lattice with near-root deletions.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs N independent replicas (one process per GPU, launched by
torch.distributed.run); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--batch-ops", type=int, default=10_000)
    p.add_argument("--insert-fraction", type=float, default=0.7)
    p.add_argument("--roots", type=int, default=64)
    p.add_argument("--check-batches", type=int, default=8)
    p.add_argument("--ref-batches", type=int, default=20,
                   help="batches of each stream checked bit-exactly against the CPU reference after every batch")
    p.add_argument("--cpu-seconds", type=float, default=20.0, help="bound of the CPU-baseline sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the lognormal and grid stream measurements")
    p.add_argument("--seed", type=int, default=22)
    p.add_argument("--alpha", type=float, default=None, help="fix the direction switch (skips the autotune sweep)")
    p.add_argument("--beta", type=float, default=None)
    return p.parse_args()


def workload(args):
    import workloads as w

    V = 1 << args.scale
    edges = w.rmat_edges(args.scale, args.edge_factor, seed=args.seed)
    roots = w.non_isolated_roots(edges, V, args.roots, seed=args.seed + 1)
    nb = 2 * (args.warmup + args.steps) + args.check_batches
    stream = w.mixed_stream(edges, V, [args.batch_ops] * nb, args.insert_fraction, seed=args.seed + 2)
    return V, edges, roots, stream


def vx_roots(roots, k, V, edges, args):
    """k seeded non-isolated roots (the first len(roots) are the single-root ones)."""
    import workloads as w

    if k <= len(roots):
        return roots[:k]
    return w.non_isolated_roots(edges, V, k, seed=args.seed + 1)


def config_dict(args, V):
    return {
        "workload": f"rmat{args.scale}-undirected-ef{args.edge_factor}-incremental-bfs-{args.batch_ops}-op-batches",
        "vertices": V,
        "edge_factor": args.edge_factor,
        "rmat": [0.57, 0.19, 0.19],
        "batch_ops": args.batch_ops,
        "insert_fraction": args.insert_fraction,
        "bfs_roots": args.roots,
        "dist": "uint32",
        "l2": "inputs larger than L2 (base CSR ~0.5 GB per step read set)",
        "parallelism": f"replicas{args.gpus}",
    }


class ClockSampler:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """DRAM bytes per full-BFS launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "bfs_full_rmat22_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def profiled_step_traffic():
    """DRAM bytes per update step from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "update_step_rmat22_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


# ----------------------------------------------------------------- B200 arm --

def run_b200(args, rank, world, local):
    import torch

    torch.cuda.set_device(local)
    from velographx_b200 import replicas

    dist = None
    if world > 1:
        import torch.distributed as dist

        replicas.init("nccl", timeout_s=120.0)

    def barrier_max(x: float) -> float:
        return replicas.max_over_ranks(x, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()

    import velographx_b200 as vx

    V, edges, roots, stream = workload(args)
    g = vx.Graph(V, False)
    g.bulk_load_edges(edges)
    # device memory for every batch of the run reserved up front (no batch
    # allocates, and so synchronises, inside a timed region)
    g.reserve(args.batch_ops, args.batch_ops * stream.batches)
    cs = torch.cuda.ExternalStream(g.stream)
    A = g.edge_count_directed()

    # ---- the library's autotuner picks the direction switch and the
    # grid-expanded row length on a few roots (untimed) ----
    tuner = vx.IncrementalBFS(g, int(roots[0]))
    if args.alpha is not None and args.beta is not None:
        tuner.set_tuning(args.alpha, args.beta, 1024)
        chosen = {"alpha": args.alpha, "beta": args.beta, "large_row": 1024, "fixed": True}
    else:
        chosen = tuner.autotune(roots[: min(16, len(roots))])
    alpha, beta, large_row = tuner.tuning()
    del tuner

    # ---- direction-optimising full BFS from the roots (GTEPS, roofline) ----
    bfs_ms, arcs, levels = [], [], []
    trace = None
    for r in roots.tolist():
        b = vx.IncrementalBFS(g, int(r))
        b.set_tuning(alpha, beta, large_row)
        b.recompute()  # warm
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record(cs)
        b.recompute()
        s1.record(cs)
        s1.synchronize()
        bfs_ms.append(s0.elapsed_time(s1))
        arcs.append(b.reached_arcs())
        levels.append(b.stats()["levels"])
        if trace is None:
            trace = [(round(us, 1), int(nf), "BU" if bu else "TD") for us, nf, bu in b.level_trace()]
        del b
    bfs_ms = np.array(bfs_ms)
    arcs = np.array(arcs, dtype=np.float64)
    gteps = float((arcs / 2).sum() / (bfs_ms.sum() * 1e-3) / 1e9)
    b_full = 4.0 * arcs + 8.0 * (V + 1) + 4.0 * V
    achieved = float((b_full / (bfs_ms * 1e-3)).mean() / 1e9)

    # ---- multi-root BFS: 64 and 256 roots in one bit-parallel launch ----
    multiroot = {}
    for k in (64, 256):
        rr = vx_roots(roots, k, V, edges, args)
        mr = vx.MultiRootBFS(g, rr)
        mr.run()  # warm
        runs = []
        for _ in range(3):  # median of three timed runs
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s0.record(cs)
            mr.run()
            s1.record(cs)
            s1.synchronize()
            runs.append(s0.elapsed_time(s1))
        ms = float(np.median(runs))
        marcs = mr.reached_arcs()
        # bit-parallel algorithmic bytes: every level reads each row once for
        # all roots (offsets + columns) and the W frontier/visited words of
        # every vertex, plus one distance write per (root, vertex)
        W = (k + 31) // 32
        b_bitpar = mr.levels * (8.0 * (V + 1) + 4.0 * A + 2 * 4.0 * W * V) + 4.0 * k * V
        b_noshare = float((4.0 * np.asarray([marcs / max(1, k)]) + 8.0 * (V + 1) + 4.0 * V)[0]) * k
        multiroot[str(k)] = {"ms": ms, "ms_runs": [round(x, 3) for x in runs],
                             "gteps": marcs / 2 / (ms * 1e-3) / 1e9, "levels": mr.levels,
                             "level_trace_us_nf_dir": [[round(us, 1), int(nf), "pull" if pull else "push"]
                                                       for us, nf, pull in mr.level_trace()],
                             "algorithmic_bytes_bitparallel": b_bitpar,
                             "achieved_gbs_bitparallel": b_bitpar / (ms * 1e-3) / 1e9,
                             "algorithmic_bytes_no_sharing": b_noshare,
                             "achieved_gbs_no_sharing": b_noshare / (ms * 1e-3) / 1e9}
        if k == 64:  # rows of the last run against single-root full BFS (untimed)
            d = mr.distances_array()
            rows = (0, 21, 42, 63)
            multiroot[str(k)]["rows_equal_single_root"] = {
                "rows": list(rows),
                "exact": all(np.array_equal(d[r], vx.IncrementalBFS(g, int(rr[r])).distances_array())
                             for r in rows)}
            del d
        del mr

    # ---- update stream, device-resident batches (value) ----
    root = int(roots[0])
    b = vx.IncrementalBFS(g, root)
    b.set_tuning(alpha, beta, large_row)
    ops = args.batch_ops
    dsrc = torch.from_numpy(stream.src.view(np.int32)).cuda()
    ddst = torch.from_numpy(stream.dst.view(np.int32)).cuda()
    dadd = torch.from_numpy(stream.add).cuda()
    torch.cuda.synchronize()

    def dev_step(i):
        off = int(stream.offsets[i])
        b.apply_device(dsrc.data_ptr() + 4 * off, ddst.data_ptr() + 4 * off, dadd.data_ptr() + off, ops, V)

    for i in range(args.warmup):
        dev_step(i)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = vx.launch_count()
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        e0.record(cs)
        for i in range(args.warmup, args.warmup + args.steps):
            dev_step(i)
        e1.record(cs)
        torch.cuda.synchronize()
    launches = vx.launch_count() - launches0
    t_dev = barrier_max(e0.elapsed_time(e1) * 1e-3)
    barrier()
    value = world * args.steps / t_dev
    st = b.stats()

    # ---- e2e through the public API with pinned host batches ----
    base = args.warmup + args.steps
    pin = torch.empty(stream.src.size * 9, dtype=torch.uint8, pin_memory=True).numpy()
    hs = pin[: 4 * stream.src.size].view(np.uint32)
    hd = pin[4 * stream.src.size: 8 * stream.src.size].view(np.uint32)
    ha = pin[8 * stream.src.size:]
    hs[:], hd[:], ha[:] = stream.src, stream.dst, stream.add

    def host_step(i):
        lo, hi = int(stream.offsets[i]), int(stream.offsets[i + 1])
        b.apply_arrays(hs[lo:hi], hd[lo:hi], ha[lo:hi])
        return b.stats()

    for i in range(base, base + args.warmup):
        host_step(i)
    torch.cuda.synchronize()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(cs)
    readback = 0
    for i in range(base + args.warmup, base + args.warmup + args.steps):
        readback = host_step(i)["readback_bytes"]
    h1.record(cs)
    torch.cuda.synchronize()
    t_e2e = barrier_max(h0.elapsed_time(h1) * 1e-3)

    # ---- exactness: repair vs fresh full BFS after each checked batch ----
    exact = True
    chk0 = base + args.warmup + args.steps
    for i in range(chk0, chk0 + args.check_batches):
        lo, hi = int(stream.offsets[i]), int(stream.offsets[i + 1])
        b.apply_arrays(stream.src[lo:hi], stream.dst[lo:hi], stream.add[lo:hi])
        fresh = vx.IncrementalBFS(g, root)
        same = np.array_equal(b.distances_array(), fresh.distances_array())
        exact = exact and same and b.reachable_count == fresh.reachable_count
        del fresh

    # ---- the records of the first ref_batches batches on a fresh replica
    # (untimed), for the per-batch comparison with the CPU reference ----
    # The same replica counts the algorithmic bytes of the timed batches
    # (batches warmup .. warmup + steps - 1, the ones the timed region
    # applied): the update launch's own accounting (vx_bfs_set_accounting)
    # for the repair and commit, plus the batch's arrays and canonical arcs.
    gpu_recs = []
    acct = None
    from workloads.streams import record

    gv = vx.Graph(V, False)
    gv.bulk_load_edges(edges)
    gv.reserve(args.batch_ops, args.batch_ops * stream.batches)
    bv = vx.IncrementalBFS(gv, root)
    bv.set_tuning(alpha, beta, large_row)
    want_recs = args.ref_batches if (rank == 0 and world == 1 and not args.no_cpu) else 0
    for i in range(max(want_recs, args.warmup + args.steps)):
        if i == args.warmup:
            bv.set_accounting(True)
        lo, hi = int(stream.offsets[i]), int(stream.offsets[i + 1])
        bv.apply_device(dsrc.data_ptr() + 4 * lo, ddst.data_ptr() + 4 * lo, dadd.data_ptr() + lo, hi - lo, V)
        if i == args.warmup + args.steps - 1:
            acct = bv.accounting()
            bv.set_accounting(False)
        if i < want_recs:
            gpu_recs.append(record(gv, bv))
    del bv, gv

    hbm, hbm_kind = measured_hbm()
    traffic = profiled_traffic()
    # bytes one update step must move at least (per batch): the op arrays the
    # canonicalisation reads (9 B per op), its canonical arcs written and read
    # back (17 B each: u, v, flags, base position), the delta-row entries the
    # commit reads and writes (4 B), and the repair's row arcs and visited
    # vertices (4 B each: a column id, a distance)
    nb_acct = max(1, acct["batches"])
    step_bytes = (9.0 * args.batch_ops + 2 * 17.0 * acct["canonical_arcs"] / nb_acct
                  + 4.0 * acct["delta_entries"] / nb_acct + 4.0 * acct["arcs_scanned"] / nb_acct
                  + 4.0 * acct["vertices_visited"] / nb_acct)
    step_achieved = step_bytes / (t_dev / args.steps) / 1e9
    step_traffic = profiled_step_traffic()
    line = {
        "metric": "update-batches/s",
        "value": value,
        "unit": "batches/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_dev * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded R-MAT and update stream)",
        "config": config_dict(args, V),
        "exact": bool(exact),
        "exact_checked_batches": args.check_batches,
        "e2e": {"value": world * args.steps / t_e2e, "unit": "batches/s",
                "h2d_bytes_per_step": ops * 9, "d2h_bytes_per_step": int(readback)},
        "gpu_launches": int(launches),
        "roofline": {
            "kernel": "bfs_full_kernel (full direction-optimising BFS)",
            "bound": "hbm",
            "achieved": achieved,
            "peak": hbm,
            "peak_kind": hbm_kind,
            "unit": "GB/s",
            "frac": achieved / hbm,
            "traffic": (traffic or {}).get("dram_bytes_per_launch"),
            "algorithmic_bytes": "4*A_r + 8*(V+1) + 4*V per root",
            # the DRAM bytes ncu counts per launch over the median launch time
            "frac_dram_traffic": (((traffic or {}).get("dram_bytes_per_launch") or 0)
                                  / (float(np.median(bfs_ms)) * 1e-3) / 1e9 / hbm) if traffic else None,
        },
        "roofline_step": {
            "kernel": "one update step: canon_cluster_kernel + bfs_stream_kernel (fused commit and repair)",
            "bound": "hbm",
            "achieved": step_achieved,
            "peak": hbm,
            "peak_kind": hbm_kind,
            "unit": "GB/s",
            "frac": step_achieved / hbm,
            "algorithmic_bytes_per_batch": step_bytes,
            "traffic": (step_traffic or {}).get("dram_bytes_per_batch"),
            "frac_dram_traffic": (((step_traffic or {}).get("dram_bytes_per_batch") or 0) / (t_dev / args.steps)
                                  / 1e9 / hbm) if step_traffic else None,
            "counters_per_batch": {k: acct[k] / nb_acct for k in ("arcs_scanned", "vertices_visited",
                                                                  "delta_entries", "canonical_arcs")},
            "algorithmic_bytes": "9*ops + 2*17*canonical_arcs + 4*delta_entries + 4*arcs_scanned + "
                                 "4*vertices_visited per batch (counted by the launch on a replica)",
        },
        "bfs": {"roots": int(len(roots)), "gteps": gteps, "ms_mean": float(bfs_ms.mean()),
                "ms_median": float(np.median(bfs_ms)), "levels_median": float(np.median(levels)),
                "arcs": int(A), "level_trace_root0_us_nf_dir": trace,
                "autotune": {"alpha": alpha, "beta": beta, "large_row": int(large_row), "chosen": chosen,
                             "by": "vx_bfs_autotune (36 candidates, mean over 16 roots of the faster of two runs)"}},
        "multiroot_bfs": multiroot,
        "repair_last": {"affected": st["last_affected_vertices"], "candidates": st["last_deletion_candidates"],
                        "full": st["last_used_full_recompute"]},
        "clocks": clocks.summary(),
    }
    if world == 1 and not args.no_extras:
        # the other stream configurations, end to end (not part of the timed region above)
        from workloads import streams as sbm

        del b
        torch.cuda.synchronize()
        c1 = sbm.insertions_c1()
        ln = sbm.lognormal(20, batches=1000, check_batches=100)
        gr = sbm.grid(4096, batches=500, check_every=100, ref_batches=args.ref_batches)
        line["streams"] = {"insertions_rmat14": c1, "lognormal_rmat20": ln, "grid4096_near_root": gr}
        checks = {k: v.pop("_check", None) for k, v in line["streams"].items()}
        roots20 = ln.pop("_roots", None)
        if rank == 0 and not args.no_cpu:
            for name, rec_samples in (("insertions_rmat14", 5), ("lognormal_rmat20", 2), ("grid4096_near_root", 1)):
                if checks[name] is not None:
                    ce, cst, croot, crecs = checks[name]
                    line["streams"][name]["cpu_baseline"] = reference_check(
                        ce, line["streams"][name]["vertices"], croot, cst, crecs, rec_samples)
            if roots20 is not None:
                ln["multiroot"]["cpu_baseline"] = reference_multiroot(checks["lognormal_rmat20"][0], roots20)
        del checks
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args, V, edges, roots, stream, gpu_recs)
        line["exact_vs_reference"] = dict(line["cpu_baseline"].get("exact_vs_reference", {}))
        line["host"] = host_info()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------- reference CPU path --

def reference_stream(args, V, edges, root, stream, first, count, budget_s):
    """Times the reference IncrementalBFS::apply (oracle/_ref, single-threaded
    like the reference) on batches [first, first+count) after replaying
    [0, first) untimed.  Returns (batches timed, seconds)."""
    from oracle import OracleBFS, OracleGraph

    g = OracleGraph(V, False, "reference")
    g.bulk_load_edges(edges)
    b = OracleBFS(g, root)
    for i in range(first):
        b.apply(*stream.batch(i))
    done, t = 0, 0.0
    for i in range(first, first + count):
        s, d, a = stream.batch(i)
        t0 = time.perf_counter()
        b.apply(s, d, a)
        t += time.perf_counter() - t0
        done += 1
        if t > budget_s:
            break
    return done, t


def host_info() -> dict:
    """The host's core count and CPU model (the CPU baseline runs there)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


def reference_check(edges, V, root, stream, gpu_recs, recompute_samples=1, budget_s=None):
    """The reference's IncrementalBFS::apply (oracle/_ref, single-threaded, as
    the reference path is) on the first len(gpu_recs) batches of the stream,
    each batch's post-batch state compared with the GPU's record; then
    recompute() timed recompute_samples times (the full arm of every batch)."""
    from oracle import available
    from oracle.replay import BatchRecord, Replay, mismatch

    if not available("reference"):
        return {"value": None, "unavailable": "oracle/_ref not built"}
    rp = Replay(edges, V, root, kind="reference")
    t, n, bad = 0.0, 0, []
    for i, rec in enumerate(gpu_recs):
        t += rp.apply_timed(*stream.batch(i))
        n += 1
        why = mismatch(BatchRecord(*rec), rp.record(), V, rp.fraction)
        if why:
            bad.append(f"batch {i}: {why}")
        if budget_s is not None and t > budget_s:
            break
    rec_s = [rp.recompute_timed() for _ in range(recompute_samples)]
    return {"value": n / t if t > 0 else None, "unit": "batches/s", "cores": 1, "kind": "reference",
            "sample": f"IncrementalBFS::apply on the first {n} batches of the same stream (single-threaded, as "
                      f"the reference path is), each checked against the GPU",
            "recompute_ms": float(np.median(rec_s)) * 1e3,
            "recompute_sample": f"IncrementalBFS::recompute, {recompute_samples} run(s), single-threaded",
            "exact_vs_reference": {"batches": n, "exact": not bad, "first_mismatch": bad[:1]}}


def reference_multiroot(edges, roots):
    """The reference's multicore path for many roots: thread-per-root
    bfs_distances over all host cores (benchmarks/thread_scaling_bfs.cpp:78-108)."""
    from oracle import available, csr_multi_bfs

    if not available("reference"):
        return {"value": None, "unavailable": "oracle/_ref not built"}
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    _, arcs, _ = csr_multi_bfs(edges, roots, cores)
    tb = time.perf_counter() - t0
    return {"value": float(arcs.sum() / 2 / tb / 1e9), "unit": "GTEPS", "cores": cores, "kind": "reference",
            "ms": tb * 1e3, "sample": f"thread-per-root bfs_distances over {len(roots)} roots on {cores} threads"}


def cpu_baseline(args, V, edges, roots, stream, gpu_recs):
    from oracle import available

    if not available("reference"):
        return {"value": None, "unit": "batches/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    out = reference_check(edges, V, int(roots[0]), stream, gpu_recs, recompute_samples=2,
                          budget_s=args.cpu_seconds)
    mr = reference_multiroot(edges, roots)
    out["bfs_gteps"] = mr["value"]
    out["bfs_sample"] = mr["sample"]
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    V, edges, roots, stream = workload(args)
    from oracle import available

    if not available("reference"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvxref.so is not built"}))
        return
    w, k = args.warmup, args.steps
    # warm-up batches are replayed untimed, then k batches timed (same batches as the B200 arm)
    n, t = reference_stream(args, V, edges, int(roots[0]), stream, w, k, 1e9)
    value = n / t
    print(json.dumps({
        "impl": "reference", "metric": "update-batches/s", "value": value, "unit": "batches/s", "n_gpus": world,
        "steps": n, "warmup": w, "ms_per_step": t * 1e3 / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded R-MAT and update stream)",
        "config": config_dict(args, V),
        "cpu_baseline": {"value": value, "unit": "batches/s", "cores": 1, "kind": "reference",
                         "sample": f"IncrementalBFS::apply, batches {w}..{w + n - 1} of the stream"},
        "e2e": {"value": value, "unit": "batches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "host": host_info(),
    }), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if args.gpus == 1 else 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world, local)


if __name__ == "__main__":
    main()
