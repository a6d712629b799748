"""sygraph_b200: SYgraph's frontier hot path on NVIDIA B200 (sm_100a).

The compute path is libsygraph_b200.so (hand-written CUDA behind a C ABI,
include/sygraph_b200.h).  This package is its Python mirror, laid out like
the reference's namespaces:

    formats.CSR, io.fromBinary / toBinary / fromMM / fromMatrix / rmat / grid,
    graph.build.fromCSR, frontier.makeFrontier / swap,
    operators.advance / filter / compute / intersection,
    algorithms.BFS / SSSP / CC / BC / TC.

Importing it requires the built library; there is no CPU fallback.
"""
from __future__ import annotations

import types as _types

from . import _lib  # noqa: F401  (raises ImportError when the library is missing)
from . import algorithms, io
from .core import (GRAPH_DIRECTED, GRAPH_WEIGHTED, WEIGHT_F32, WEIGHT_NONE, WEIGHT_U32, CSR, DeviceArray, Frontier,
                   Graph, Properties, build, device_count, launch_count, makeFrontier, swap)

formats = _types.SimpleNamespace(CSR=CSR)
graph = _types.SimpleNamespace(build=build, Graph=Graph, Properties=Properties)
frontier = _types.SimpleNamespace(makeFrontier=makeFrontier, swap=swap, Frontier=Frontier)

try:  # the operator layer binds entry points that may be absent from an older build
    from . import operators  # noqa: F401
except ImportError:  # pragma: no cover
    operators = None

__all__ = ["CSR", "DeviceArray", "Frontier", "Graph", "Properties", "algorithms", "build", "device_count", "formats",
           "frontier", "graph", "io", "launch_count", "makeFrontier", "operators", "swap", "WEIGHT_F32", "WEIGHT_NONE",
           "WEIGHT_U32", "GRAPH_DIRECTED", "GRAPH_WEIGHTED"]
