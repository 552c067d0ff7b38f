"""CPU oracle for the dynamic-BFS path (test infrastructure only).

Two interchangeable back ends with one Python surface:

* ``kind="port"``      -- ``liboracle.so``, the plain-C restatement in
  ``vx_oracle.c`` (always available once ``make -C oracle`` ran);
* ``kind="reference"`` -- ``_ref/libvxref.so``, the unmodified VeloGraphX
  ``DynamicGraph`` / ``IncrementalBFS`` compiled from the reference headers.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package.  The product never does.
"""
from .oracle import (  # noqa: F401
    UNREACHABLE,
    OracleBFS,
    OracleGraph,
    available,
    build,
    csr_multi_bfs,
    load,
)
