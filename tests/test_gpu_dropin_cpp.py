"""GPU: the reference's own C++ tests of this path, compiled unchanged against
this repository's drop-in headers (include/velographx/...) and linked to
libvx_b200.so by oracle/Makefile's ``dropin`` target, run green:

* tests/test_incremental_bfs_deletion.cpp -- every microcase and the 250-epoch
  randomized stream compare IncrementalBFS::apply with a fresh recompute;
* tests/test_incremental_components_deletion.cpp -- IncrementalComponents
  across a deletion and a mixed batch (partition and last_repaired_vertices);
* tests/test_io.cpp -- io::save_binary / io::load_binary round trip;
* tests/test_io_hardening.cpp -- load_edge_list: comments, blank lines, and
  the malformed / trailing-data / uint32-overflow errors with their types.
"""
import os
import subprocess
import tempfile

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


@pytest.mark.parametrize("name", ["test_incremental_bfs_deletion", "test_incremental_components_deletion", "test_io",
                                  "test_io_hardening"])
def test_reference_cpp_suite_runs_on_the_gpu_library(name):
    binary = os.path.join(REF, "dropin_" + name)
    if not os.path.exists(binary):
        pytest.skip("drop-in build not present (needs the reference tree at build time)")
    with tempfile.TemporaryDirectory() as cwd:  # test_io writes its file into the working directory
        r = subprocess.run([binary], capture_output=True, text=True, timeout=600, cwd=cwd)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    assert "libvx_b200.so" in subprocess.run(["ldd", binary], capture_output=True, text=True).stdout
