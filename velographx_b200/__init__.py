"""VeloGraphX dynamic-BFS path on NVIDIA B200.

Drop-in for the dynamic-BFS part of the reference's ``velographx`` module
(python/bindings.cpp:38-52): ``UpdateBatch``, ``Graph``, ``IncrementalBFS``,
``from_numpy_edges``, ``from_scipy_csr``, ``from_arrow_columns`` and
``from_arrow_table``.  Everything runs on the GPU through ``libvx_b200.so``;
there is no host fallback -- importing fails loudly when the native library
has not been built.
"""
from __future__ import annotations

import ctypes as _ctypes
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_HERE, "libvx_b200.so")

try:
    from ._velographx import (  # noqa: F401
        Graph,
        IncrementalBFS,
        IncrementalComponents,
        IncrementalSSSP,
        MultiRootBFS,
        UpdateBatch,
        from_arrow_columns,
        from_arrow_table,
        from_numpy_edges,
        from_scipy_csr,
        last_error,
        launch_count,
        consolidate_to_csr_snapshot,
        load_binary,
        load_edge_list,
        neighbor_scan_ns,
        save_binary,
    )
except ImportError as exc:  # pragma: no cover - exercised only on a broken install
    raise ImportError(
        "velographx_b200: the native extension is not built (run __graft_entry__.build() "
        "or python velographx_b200/build.py): " + str(exc)
    ) from exc

_capi = None


def capi() -> _ctypes.CDLL:
    """The C ABI of include/vx_b200.h as a ctypes library (same .so the module uses)."""
    global _capi
    if _capi is None:
        _capi = _ctypes.CDLL(LIB_PATH)
    return _capi


__all__ = [
    "Graph",
    "IncrementalBFS",
    "IncrementalComponents",
    "IncrementalSSSP",
    "MultiRootBFS",
    "UpdateBatch",
    "from_numpy_edges",
    "from_scipy_csr",
    "from_arrow_columns",
    "from_arrow_table",
    "load_edge_list",
    "save_binary",
    "load_binary",
    "capi",
    "LIB_PATH",
]
