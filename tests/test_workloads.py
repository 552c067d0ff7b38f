"""CPU: the seeded generators are deterministic and have the configured shapes."""
import numpy as np

import workloads as w


def test_rmat_deterministic_and_skewed():
    a = w.rmat_edges(12, seed=3)
    b = w.rmat_edges(12, seed=3)
    assert a.shape == (16 << 12, 2) and np.array_equal(a, b)
    assert not np.array_equal(a, w.rmat_edges(12, seed=4))
    deg = np.bincount(a.ravel(), minlength=1 << 12)
    assert deg.max() > 20 * deg.mean()  # heavy-tailed (a = 0.57)
    assert a.max() < (1 << 12)


def test_grid_shape():
    g = w.grid_edges(8, 8, long_range_fraction=0.0)
    assert g.shape == (2 * 8 * 7, 2)
    assert set(map(tuple, g[:3].tolist())) == {(0, 1), (1, 2), (2, 3)}
    g2 = w.grid_edges(64, 64, 0.001)
    assert g2.shape[0] == 2 * 64 * 63 + round(2 * 64 * 63 * 0.001)


def test_streams():
    e = w.rmat_edges(10, seed=1)
    st = w.mixed_stream(e, 1024, [10, 20, 30], 0.7, seed=2)
    assert st.batches == 3 and st.src.size == 60
    s, d, a = st.batch(1)
    assert s.size == 20
    sizes = w.lognormal_sizes(1000)
    assert sizes.min() >= 1 and sizes.max() <= 200_000 and 300 < np.median(sizes) < 800
    roots = w.non_isolated_roots(e, 1024, 16)
    assert roots.size == 16 and len(set(roots.tolist())) == 16


def test_generators_byte_identical_to_recorded_outputs():
    """The generators moved out of the GPU library into workloads/gen.c; the
    edge arrays must stay byte-identical to the recorded ones (sha256 prefixes
    taken from the earlier in-library generators)."""
    import hashlib

    def h(a):
        return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:32]

    assert h(w.rmat_edges(14, seed=1)) == "59f562230e9d1cb7c4bbceee04e7e837"
    assert h(w.rmat_edges(12, seed=12)) == "1db7b9080a24f4f82a4913951a279c08"
    assert h(w.rmat_edges(16, 8, 0.45, 0.15, 0.15, seed=5)) == "7214bb59a3830418a9f742474ed387c0"
    assert h(w.uniform_edges(1000003, 100000, seed=3)) == "20e42664c7cc0a20562422c982e21297"
    assert h(w.grid_edges(64, 80, 0.01, seed=4)) == "859484fca67739efc31c7981d3710c1d"


def test_workloads_do_not_load_the_gpu_library():
    """The benchmark's reference arm builds its inputs with this package; it
    must not load libvx_b200.so (checked in a fresh interpreter)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, workloads as w, oracle; w.rmat_edges(10, seed=1); "
            "maps = open('/proc/self/maps').read(); "
            "sys.exit(1 if ('libvx_b200' in maps or 'velographx_b200' in sys.modules) else 0)")
    assert subprocess.run([sys.executable, "-c", code], cwd=root).returncode == 0


def test_digest_matches_definition():
    d = np.array([0, 1, 0xFFFFFFFF, 7], dtype=np.uint32)
    M = (1 << 64) - 1

    def mix(z):
        z = (z + 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    assert w.digest(d) == sum(mix((v << 32) | int(x)) for v, x in enumerate(d)) & M
