"""The 9-regime selector study (benchmark harness, not the product).

The reference chooses, per update batch, between ``IncrementalBFS.apply``
(repair) and ``graph.apply`` + ``recompute`` (full) in its benchmark harnesses
(benchmarks/publication_policy_bfs.cpp:46-335) with a hand-tuned heuristic;
regret is measured offline against the per-batch oracle
min(t_repair, t_full), full winning ties (tools/summarize_publication_policy.py:66,72).

* ``collect`` runs a regime's stream on two graph replicas in lockstep -- one
  executes the repair arm, the other the full arm -- so every batch carries
  its 16 device-computed features and both arms' GPU times (CUDA events on the
  graph's stream), and the two replicas' distances are compared bit for bit;
* ``evaluate`` trains ``velographx_b200.selector.MLPSelector`` on the first
  part of every regime and replays the held-out batches through the
  selectors -- the network, the network with online residual calibration,
  the reference's heuristic, and the two trivial policies of the reference's
  ablation (always repair, always full; PAPER.md:126-132) -- reporting regret
  and wrong-arm rates.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

import workloads as w
from velographx_b200 import Graph, IncrementalBFS
from velographx_b200.selector import N_FEATURES, Heuristic, MLPSelector, _check, _f32p, _lib, _u8p, _u32p


@dataclass
class RegimeData:
    name: str
    vertices: int
    features: np.ndarray
    t_repair: np.ndarray  # us
    t_full: np.ndarray  # us
    update_fraction: np.ndarray
    shallow_fraction: np.ndarray
    affected_fraction: np.ndarray
    initial_full_us: float
    initial_reachable_fraction: float
    exact: bool
    extra: dict = field(default_factory=dict)


def collect(name: str, edges: np.ndarray, vertices: int, root: int, sizes, insert_fraction: float, seed: int,
            fallback_fraction: float = 2.0, check_every: int = 1) -> RegimeData:
    """Runs the stream on two replicas (repair arm / full arm) and records
    features and both arms' GPU times for every batch."""
    import torch

    lib = _lib()
    gA, gB = Graph(vertices, False), Graph(vertices, False)
    gA.bulk_load_edges(edges)
    gB.bulk_load_edges(edges)
    # the reference harness disables the internal fallback (fraction 2.0) so
    # the selector alone owns recomputation (publication_policy_bfs.cpp:59)
    bA = IncrementalBFS(gA, root, fallback_fraction)
    bB = IncrementalBFS(gB, root, fallback_fraction)
    sA = torch.cuda.ExternalStream(gA.stream)
    sB = torch.cuda.ExternalStream(gB.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(sB)
    bB.recompute()
    e1.record(sB)
    e1.synchronize()
    initial_full_us = e0.elapsed_time(e1) * 1e3
    reach0 = bA.reachable_count / max(1, vertices)
    stream = w.mixed_stream(edges, vertices, sizes, insert_fraction, seed=seed)
    n = stream.batches
    feats = np.zeros((n, N_FEATURES), np.float32)
    t_rep = np.zeros(n)
    t_full = np.zeros(n)
    upd = np.zeros(n)
    shallow = np.zeros(n)
    aff = np.zeros(n)
    prev_aff = 0.0
    exact = True
    f16 = np.zeros(N_FEATURES, np.float32)
    for i in range(n):
        s, d, a = (np.ascontiguousarray(x) for x in stream.batch(i))
        edges_now = gA.edge_count_directed()
        upd[i] = len(s) / max(1, edges_now)
        # features of the staged batch (pre-batch state, identical on both replicas)
        _check(lib.vx_bfs_stage(C.c_void_p(bA.handle), s.ctypes.data_as(_u32p), d.ctypes.data_as(_u32p),
                                a.ctypes.data_as(_u8p), len(s)))
        _check(lib.vx_bfs_staged_features(C.c_void_p(bA.handle), prev_aff, f16.ctypes.data_as(_f32p)))
        feats[i] = f16
        if i == 0:
            shallow[i] = shallow_parent_deletion_fraction(s, d, a, bA.distances_array())
        # repair arm on A (staging already done; it is common to both arms and
        # timed separately on B below, so both times include it)
        torch.cuda.synchronize()
        e0.record(sB)
        _check(lib.vx_bfs_stage(C.c_void_p(bB.handle), s.ctypes.data_as(_u32p), d.ctypes.data_as(_u32p),
                                a.ctypes.data_as(_u8p), len(s)))
        e1.record(sB)
        e1.synchronize()
        t_stage = e0.elapsed_time(e1) * 1e3
        e0.record(sA)
        _check(lib.vx_bfs_run_repair(C.c_void_p(bA.handle)))
        e1.record(sA)
        e1.synchronize()
        t_rep[i] = t_stage + e0.elapsed_time(e1) * 1e3
        e0.record(sB)
        _check(lib.vx_bfs_run_full(C.c_void_p(bB.handle)))
        e1.record(sB)
        e1.synchronize()
        t_full[i] = t_stage + e0.elapsed_time(e1) * 1e3
        bA.mark_stale()
        bB.mark_stale()
        st = bA.stats()
        prev_aff = st["last_affected_vertices"] / max(1, vertices)
        aff[i] = prev_aff
        if check_every and i % check_every == 0:
            exact = exact and _same_distances(bA, bB)
    return RegimeData(name, vertices, feats, t_rep, t_full, upd, shallow, aff, initial_full_us, reach0, exact)


def shallow_parent_deletion_fraction(src, dst, add, dist, depth: int = 3) -> float:
    """Deletions of a shortest-parent arc at depth <= 3, both directions of an
    undirected graph, over the raw op count (adaptive_policy_bfs.cpp:126-147);
    the heuristic reads it on the first batch only."""
    unreachable = np.uint32(0xFFFFFFFF)
    rm = add == 0
    u = src[rm].astype(np.int64)
    v = dst[rm].astype(np.int64)
    ok = (u < dist.size) & (v < dist.size)
    du = dist[u[ok]]
    dv = dist[v[ok]]
    both = (du != unreachable) & (dv != unreachable)
    du64, dv64 = du.astype(np.int64), dv.astype(np.int64)
    fwd = both & (du64 + 1 == dv64) & (dv64 <= depth)
    bwd = both & (dv64 + 1 == du64) & (du64 <= depth)
    return float(fwd.sum() + bwd.sum()) / max(1, len(src))


class _DeviceU32:
    """A device array of uint32 seen by torch through __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3,
                                         "strides": None}


def _same_distances(a: IncrementalBFS, b: IncrementalBFS) -> bool:
    """Bit-for-bit comparison of two BFS distance arrays, on the device."""
    import torch

    pa, na = a.distances_device_ptr()
    pb, nb = b.distances_device_ptr()
    if na != nb:
        return False
    if na == 0:
        return True
    ta = torch.as_tensor(_DeviceU32(pa, na), device="cuda")
    tb = torch.as_tensor(_DeviceU32(pb, nb), device="cuda")
    torch.cuda.synchronize()
    return bool(torch.equal(ta, tb))


def regret(t_chosen, t_repair, t_full):
    oracle = np.minimum(t_repair, t_full)
    return np.maximum(0.0, (t_chosen - oracle) / oracle)


def calibrated_choices(pred_log: np.ndarray, ok: np.ndarray, t_repair, t_full, fallback,
                       alpha: float = 0.25) -> np.ndarray:
    """Online residual calibration of the network's predictions.

    After each batch the time of the arm that ran is observed; an EMA of the
    log-space residual (observed - predicted) of that arm is added to its
    later predictions, so a drift the network never saw in training (the graph
    grows, the machine slows) moves the decision instead of repeating the same
    mistake.  The EMA weight is the heuristic's (adaptive_policy_bfs.cpp:31).
    A non-finite prediction takes the fallback's choice for that batch."""
    res = np.zeros(2)
    seen = np.zeros(2, bool)
    out = np.zeros(len(pred_log), bool)
    for j in range(len(pred_log)):
        if not ok[j]:
            full = bool(fallback[j])
        else:
            p = pred_log[j] + res
            full = bool(p[1] <= p[0])
        out[j] = full
        if ok[j]:
            arm = 1 if full else 0
            obs = np.log(t_full[j] if full else t_repair[j])
            r = obs - pred_log[j, arm]
            res[arm] = (1 - alpha) * res[arm] + alpha * r if seen[arm] else r
            seen[arm] = True
    return out


def _summary(regrets, wrong, total, **extra):
    cat = np.concatenate(regrets)
    return {"equal_regime_mean_regret": float(np.mean([r.mean() for r in regrets])),
            "sample_weighted_regret": float(cat.mean()), "p95_regret": float(np.percentile(cat, 95)),
            "max_regret": float(cat.max()), "wrong_arm_rate": wrong / max(1, total), **extra}


def evaluate(regimes: list[RegimeData], train_fraction: float = 0.3, seed: int = 1, epochs: int = 300,
             calib_fraction: float = 1 / 3) -> dict:
    """Trains on the first train_fraction of every regime (pooled; the last
    calib_fraction of each regime's prefix is kept out of the fit and
    calibrates the decision margin, so the margin is chosen on batches the
    network has not seen, later in the stream than the ones it was fitted on)
    and compares on the rest: "mlp" (the network; the heuristic's choice where a
    prediction is not finite), "mlp_online" (the network with online residual
    calibration, an ablation), "heuristic" (the reference's adaptive
    selector, replayed online), and the two trivial policies of the
    reference's feature ablation, "always_repair" and "always_full"
    (PAPER.md:126-132)."""
    tr_X, tr_r, tr_f, ca_X, ca_r, ca_f = [], [], [], [], [], []
    for rg in regimes:
        k = max(1, int(len(rg.t_repair) * train_fraction))
        c = min(k - 1, int(k * calib_fraction))  # the prefix's last c batches calibrate
        tr_X.append(rg.features[:k - c])
        tr_r.append(rg.t_repair[:k - c])
        tr_f.append(rg.t_full[:k - c])
        ca_X.append(rg.features[k - c:k])
        ca_r.append(rg.t_repair[k - c:k])
        ca_f.append(rg.t_full[k - c:k])
    calib = (np.concatenate(ca_X), np.concatenate(ca_r), np.concatenate(ca_f))
    mlp = MLPSelector(seed)
    loss = mlp.fit(np.concatenate(tr_X), np.concatenate(tr_r), np.concatenate(tr_f), epochs=epochs, seed=seed,
                   calib=calib if len(calib[0]) else None)
    out = {"train_loss": loss, "margin": float(mlp.margin), "calib_fraction": calib_fraction, "regimes": {}}
    names = ("mlp", "mlp_online", "heuristic", "always_repair", "always_full")
    regrets = {n: [] for n in names}
    wrong = dict.fromkeys(names, 0)
    total = 0
    fallbacks = 0
    for rg in regimes:
        k = max(1, int(len(rg.t_repair) * train_fraction))
        X = rg.features[k:]
        tr, tf = rg.t_repair[k:], rg.t_full[k:]
        oracle_full = tf <= tr
        # heuristic replayed online with the measured time of the arm it picks
        h = Heuristic(rg.vertices, rg.initial_reachable_fraction, rg.initial_full_us)
        for i in range(k):  # warm its EMA state on the training prefix, as the harness would
            full = h.decide(rg.update_fraction[i], rg.shallow_fraction[i])
            h.observe(full, rg.t_full[i] if full else rg.t_repair[i], 0.0 if full else rg.affected_fraction[i])
        h_full = np.zeros(len(tr), bool)
        for j in range(len(tr)):
            i = k + j
            full = h.decide(rg.update_fraction[i], rg.shallow_fraction[i])
            h_full[j] = full
            h.observe(full, tf[j] if full else tr[j], 0.0 if full else rg.affected_fraction[i])
        pred = mlp.predict_log(X)
        ok = np.all(np.isfinite(pred), axis=1)
        fallbacks += int((~ok).sum())
        static = np.where(ok, mlp.choose_full(X)[0], h_full)
        choice = {"mlp": static, "mlp_online": calibrated_choices(pred, ok, tr, tf, h_full), "heuristic": h_full,
                  "always_repair": np.zeros(len(tr), bool), "always_full": np.ones(len(tr), bool)}
        row = {"batches": len(tr), "full_share_oracle": float(oracle_full.mean()), "exact": rg.exact}
        for n in names:
            r = regret(np.where(choice[n], tf, tr), tr, tf)
            regrets[n].append(r)
            wrong[n] += int((choice[n] != oracle_full).sum())
            row[f"{n}_mean_regret"] = float(r.mean())
            row[f"{n}_wrong_arm"] = float((choice[n] != oracle_full).mean())
        out["regimes"][rg.name] = row
        total += len(tr)
    out["mlp"] = _summary(regrets["mlp"], wrong["mlp"], total, fallbacks=fallbacks)
    out["mlp_online"] = _summary(regrets["mlp_online"], wrong["mlp_online"], total)
    for n in ("heuristic", "always_repair", "always_full"):
        out[n] = _summary(regrets[n], wrong[n], total)
    out["exact"] = all(r.exact for r in regimes)
    return out


def regime_graphs(scale_rmat: int = 20, er_vertices: int = 1 << 20, grid_side: int = 2048, seed: int = 5):
    """The three graphs of the selector study: R-MAT, Erdos-Renyi (avg degree
    16), and a lattice with 0.1% random long-range edges."""
    rm = w.rmat_edges(scale_rmat, seed=seed)
    er = w.uniform_edges(er_vertices, er_vertices * 8, seed=seed + 1)
    gr = w.grid_edges(grid_side, grid_side, 0.001, seed=seed + 2)
    return [("rmat", rm, 1 << scale_rmat), ("er", er, er_vertices), ("grid", gr, grid_side * grid_side)]


_ARRAYS = ("features", "t_repair", "t_full", "update_fraction", "shallow_fraction", "affected_fraction")


def save_regimes(path: str, regimes: list[RegimeData]) -> None:
    """The collected batches (features and both arms' times) as one .npz, so
    the evaluation can be repeated without timing the arms again."""
    import json

    arrays = {f"{i}_{n}": getattr(r, n) for i, r in enumerate(regimes) for n in _ARRAYS}
    meta = [{"name": r.name, "vertices": r.vertices, "initial_full_us": r.initial_full_us,
             "initial_reachable_fraction": r.initial_reachable_fraction, "exact": r.exact} for r in regimes]
    np.savez_compressed(path, meta=np.array(json.dumps(meta)), **arrays)


def load_regimes(path: str) -> list[RegimeData]:
    import json

    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    return [RegimeData(m["name"], m["vertices"], *(z[f"{i}_{n}"] for n in _ARRAYS), m["initial_full_us"],
                       m["initial_reachable_fraction"], m["exact"]) for i, m in enumerate(meta)]


def study(batches_per_regime: int = 1111, sizes=(10, 1000, 100000), insert_fraction: float = 0.75,
          train_fraction: float = 0.3, epochs: int = 300, scale_rmat: int = 20, er_vertices: int = 1 << 20,
          grid_side: int = 2048, seed: int = 5, log=None, data: str | None = None) -> dict:
    """The 9-regime selector study: {R-MAT, Erdos-Renyi, lattice} x batch sizes,
    both arms timed on every batch, distances compared bit for bit, MLP trained
    on the first train_fraction of each regime and scored on the rest.  With
    data, the collected batches are read from that .npz when it exists and
    saved to it otherwise."""
    import os

    if data and os.path.exists(data):
        regimes = load_regimes(data)
    else:
        regimes = []
        for gname, edges, V in regime_graphs(scale_rmat, er_vertices, grid_side, seed):
            root = w.max_degree_root(edges, V)
            for k, size in enumerate(sizes):
                rd = collect(f"{gname}_{size}", edges, V, root, np.full(batches_per_regime, size), insert_fraction,
                             seed=seed * 100 + k)
                if log:
                    log(f"{rd.name}: repair median {np.median(rd.t_repair):.1f} us, full median "
                        f"{np.median(rd.t_full):.1f} us, full wins {np.mean(rd.t_full <= rd.t_repair):.2f}, "
                        f"exact {rd.exact}")
                regimes.append(rd)
        if data:
            save_regimes(data, regimes)
    rep = evaluate(regimes, train_fraction=train_fraction, epochs=epochs)
    # the same network with its margin calibrated on the batches it was fitted on (ablation)
    abl = evaluate(regimes, train_fraction=train_fraction, epochs=epochs, calib_fraction=0.0)
    rep["ablation_margin_on_fit_batches"] = {"margin": abl["margin"], "mlp": abl["mlp"],
                                             "regimes": {k: v["mlp_mean_regret"] for k, v in abl["regimes"].items()}}
    rep["config"] = {"batches_per_regime": batches_per_regime, "sizes": list(sizes),
                     "insert_fraction": insert_fraction, "train_fraction": train_fraction, "epochs": epochs,
                     "graphs": {"rmat_scale": scale_rmat, "er_vertices": er_vertices, "grid_side": grid_side},
                     "seed": seed}
    rep["medians_us"] = {r.name: {"repair": float(np.median(r.t_repair)), "full": float(np.median(r.t_full))}
                         for r in regimes}
    return rep


if __name__ == "__main__":
    import argparse
    import json
    import sys

    ap = argparse.ArgumentParser(description="selector regret study (both arms timed on the GPU)")
    ap.add_argument("--batches", type=int, default=1111, help="batches per regime")
    ap.add_argument("--sizes", type=int, nargs="+", default=[10, 1000, 100000])
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--er-vertices", type=int, default=1 << 20)
    ap.add_argument("--grid-side", type=int, default=2048)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--out", default=None)
    ap.add_argument("--data", default=None, help=".npz of the collected batches: read when present, else written")
    a = ap.parse_args()
    res = study(a.batches, tuple(a.sizes), scale_rmat=a.scale, er_vertices=a.er_vertices, grid_side=a.grid_side,
                epochs=a.epochs, log=lambda m: print(m, file=sys.stderr, flush=True), data=a.data)
    text = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    print(text)
