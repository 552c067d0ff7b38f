"""CPU: the C-ABI library loads and exports every symbol its headers declare;
the Python module exposes the reference's names.  No device calls."""
import ctypes
import os
import re

import velographx_b200 as vx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"^\s*(?:int|uint64_t|void)\s+(vx_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(vx.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_surface_matches_reference_module():
    for name in ("UpdateBatch", "Graph", "IncrementalBFS", "from_numpy_edges", "from_scipy_csr",
                 "from_arrow_columns", "from_arrow_table"):
        assert hasattr(vx, name), name
    assert vx.IncrementalBFS.unreachable == 0xFFFFFFFF
    b = vx.UpdateBatch()
    b.add(0, 1)
    b.add(1, 2, timestamp=5)
    b.remove(0, 1)
    assert len(b) == 3


def test_last_error_starts_empty_and_is_callable():
    lib = ctypes.CDLL(vx.LIB_PATH)
    buf = ctypes.create_string_buffer(64)
    lib.vx_last_error.restype = ctypes.c_int
    assert lib.vx_last_error(buf, 64) >= 0


def test_null_arguments_are_rejected_without_a_device():
    lib = ctypes.CDLL(vx.LIB_PATH)
    lib.vx_graph_vertex_count.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert lib.vx_graph_vertex_count(None, None) == -1
    buf = ctypes.create_string_buffer(128)
    lib.vx_last_error(buf, 128)
    assert b"null" in buf.value
