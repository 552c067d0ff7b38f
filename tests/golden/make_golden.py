"""Generate the golden vectors of the dynamic-BFS path from the REFERENCE itself.

Runs the unmodified VeloGraphX DynamicGraph + IncrementalBFS (oracle/_ref,
built by ``make -C oracle`` from the reference headers) on seeded scenarios
and records, after every batch, the distance vector (small cases) or its
sha256 (larger cases) plus the IncrementalBFS counters.  The scenarios mirror
the reference's own BFS tests (tests/test_incremental_bfs_deletion.cpp:57-210,
tests/test_randomized_dynamic.cpp:140-191) and configuration 1 of the
benchmark plan (R-MAT scale 14, 100 batches of 64 insertions).

Usage:  python tests/golden/make_golden.py      (writes tests/golden/*.json)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden import scenarios  # noqa: E402


def digest(d: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(d, dtype="<u4").tobytes()).hexdigest()


def run_reference(sc: dict) -> dict:
    from oracle import OracleBFS, OracleGraph

    g = OracleGraph(sc["vertices"], sc["directed"], kind="reference")
    edges = sc["edges"]
    if len(edges):
        g.bulk_load_edges(edges)
    b = OracleBFS(g, sc["source"], sc["fraction"])
    keep_full = sc["vertices"] <= 64
    rec = []

    def snap():
        d = b.distances()
        item = {"len": int(d.size), "sha256": digest(d), "stats": list(map(int, b.stats())),
                "edge_count": g.edge_count_directed(), "version": g.version, "vertex_count": g.vertex_count}
        if keep_full:
            item["dist"] = d.tolist()
        rec.append(item)

    snap()
    for src, dst, add in sc["batches"]:
        b.apply(src, dst, add)
        snap()
    out = {k: v for k, v in sc.items() if k not in ("edges", "batches")}
    out["inputs_sha256"] = scenarios.inputs_digest(sc)
    out["records"] = rec
    return out


def main() -> None:
    from oracle import available

    if not available("reference"):
        raise SystemExit("oracle/_ref/libvxref.so missing: run `make -C oracle` with the reference tree present")
    for name, sc in scenarios.all_scenarios().items():
        data = run_reference(sc)
        path = os.path.join(HERE, name + ".json")
        with open(path, "w") as f:
            json.dump(data, f, separators=(",", ":"))
        print(f"{name}: {len(data['records'])} records -> {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
