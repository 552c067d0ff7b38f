"""GPU: the reference's own C++ test of the incremental BFS
(tests/test_incremental_bfs_deletion.cpp of the reference), compiled unchanged
against this repository's drop-in headers (include/velographx/...) and linked
to libvx_b200.so by oracle/Makefile's ``dropin`` target, runs green: every
microcase and the 250-epoch randomized stream compare IncrementalBFS::apply
with a fresh recompute through the B200 path."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_test_incremental_bfs_deletion")


@pytest.mark.skipif(not os.path.exists(BIN), reason="drop-in build not present (needs the reference tree at build time)")
def test_reference_cpp_bfs_deletion_suite_runs_on_the_gpu_library():
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    maps_check = subprocess.run(["ldd", BIN], capture_output=True, text=True)
    assert "libvx_b200.so" in maps_check.stdout
