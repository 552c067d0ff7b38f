"""CPU: the consolidation policy, signal and hysteresis controller of
include/velographx/storage/consolidation.hpp make the reference's decisions
(include/velographx/storage/consolidation.hpp of the reference) on a seeded
sequence of 8,000 observations across 20 configurations.  Host arithmetic
only: the driver is compiled against each header set and the printed
decisions compared."""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("VX_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include", "velographx")) or not shutil.which("g++"),
                    reason="reference headers or g++ not present")
def test_controller_decisions_equal_reference():
    src = os.path.join(ROOT, "tests", "cpp", "controller_parity.cpp")
    outs = []
    with tempfile.TemporaryDirectory() as tmp:
        for name, inc, extra in (("ours", os.path.join(ROOT, "include"),
                                  ["-L" + os.path.join(ROOT, "velographx_b200"), "-l:libvx_b200.so",
                                   "-Wl,-rpath," + os.path.join(ROOT, "velographx_b200")]),
                                 ("ref", os.path.join(REF, "include"), [])):
            exe = os.path.join(tmp, name)
            subprocess.run(["g++", "-O1", "-std=c++20", "-I" + inc, src, "-o", exe] + extra, check=True)
            outs.append(subprocess.run([exe], capture_output=True, text=True, check=True).stdout)
    assert outs[0].count("\n") > 8000
    assert outs[0] == outs[1]
