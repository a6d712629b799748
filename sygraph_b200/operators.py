"""operators::advance / filter / compute / intersection over the C ABI.

Through the C ABI a functor is one of the built-in device functors (the
``op`` / ``pred`` / ``fn`` constants below, each restating a reference
functor); the C++ header API in include/sygraph/ takes arbitrary device
lambdas.  Functor state is passed as device pointers (DeviceArray) and
scalars."""
from __future__ import annotations

import ctypes as C
import types as _types

import numpy as np

from . import _lib
from ._lib import call
from .core import DeviceArray, Frontier, Graph


class direction:  # noqa: N801 - operators::direction (operators/config.hpp:17-21)
    push = 0
    pull = 1
    pull_all = 2


class load_balancer:  # noqa: N801 - operators::load_balancer (operators/config.hpp:10-15)
    workitem_mapped = 0
    subgroup_mapped = 1
    workgroup_mapped = 2
    bucketing = 3


class frontier_view:  # noqa: N801 - frontier::frontier_view (frontier/frontier_settings.hpp:13-18)
    graph = 0
    vertex = 1
    edge = 2
    none = 3


class size:  # noqa: N801 - frontier::size (operators/config.hpp:29-33)
    fetch_from_memory = -1
    infer_from_device = 0


OP_BFS_PUSH, OP_BFS_PULL, OP_SSSP_RELAX, OP_CC_MAX, OP_BC_FORWARD, OP_BC_BACKWARD = 0, 1, 2, 3, 4, 5
OP_COUNT_VISITS, OP_NONZERO_DEGREE, OP_BFS_VISIT_FLAG, OP_TRUE = 6, 7, 8, 9
PRED_EVEN, PRED_LESS_THAN, PRED_ITER_MARK, PRED_FLAG = 0, 1, 2, 3
FN_MARK, FN_SET_U8 = 0, 1
RED_VERTEX_ID, RED_DEGREE, RED_COUNT = 0, 1, 2


def op_args(ptrs=(), u=(), f=()) -> _lib.OpArgs:
    a = _lib.OpArgs()
    for i, p in enumerate(ptrs):
        a.p[i] = p.ptr if isinstance(p, DeviceArray) else p
    for i, x in enumerate(u):
        a.u[i] = int(x)
    for i, x in enumerate(f):
        a.f[i] = float(x)
    return a


def _frontier(G: Graph, in_: Frontier | None, out: Frontier | None, op: int, args=None,
              direction_: int = direction.push, lb: int = load_balancer.workgroup_mapped,
              in_view: int = frontier_view.vertex, out_view: int | None = None,
              expected_size: int = size.fetch_from_memory) -> None:
    """advance::frontier<Direction, Lb, InView, OutView>(G, in, out, f, expected_size)
    (operators/advance/advance.hpp:116-218)."""
    if out_view is None:
        out_view = frontier_view.vertex if out is not None else frontier_view.none
    a = args if args is not None else _lib.OpArgs()
    call("sg_advance", G.handle, in_.handle if in_ is not None else None, out.handle if out is not None else None,
         direction_, lb, in_view, out_view, op, C.byref(a), expected_size)


def _vertices(G: Graph, out: Frontier | None, op: int, args=None, lb: int = load_balancer.workgroup_mapped) -> None:
    """advance::vertices<Lb, OutView>(G, out, f) (advance.hpp:46-87): every vertex is a candidate."""
    _frontier(G, None, out, op, args, direction.push, lb, frontier_view.graph)


advance = _types.SimpleNamespace(frontier=_frontier, vertices=_vertices)


def _external(G: Graph, in_: Frontier, out: Frontier, pred: int, args=None) -> None:
    """filter::external (operators/filter/filter.hpp:41-69)."""
    a = args if args is not None else _lib.OpArgs()
    call("sg_filter_external", G.handle, in_.handle, out.handle, pred, C.byref(a))


def _inplace(G: Graph, f: Frontier, pred: int, args=None) -> None:
    """filter::inplace: removes every active vertex with pred(v)."""
    a = args if args is not None else _lib.OpArgs()
    call("sg_filter_inplace", G.handle, f.handle, pred, C.byref(a))


filter = _types.SimpleNamespace(external=_external, inplace=_inplace)  # noqa: A001


def _execute(G: Graph, f: Frontier, fn: int, args=None) -> None:
    """compute::execute<vertex> (operators/for/for.hpp:48-60)."""
    a = args if args is not None else _lib.OpArgs()
    call("sg_compute_execute", G.handle, f.handle, fn, C.byref(a))


def _reduce(G: Graph, f: Frontier, fn: int, args=None) -> int:
    """compute::reduce<vertex, plus<R>> (for.hpp:62-92); returns the sum."""
    a = args if args is not None else _lib.OpArgs()
    r = C.c_uint64()
    call("sg_compute_reduce", G.handle, f.handle, fn, C.byref(a), C.byref(r))
    return r.value


compute = _types.SimpleNamespace(execute=_execute, reduce=_reduce)


def _intersect(G: Graph, in1: Frontier, in2: Frontier, out: Frontier) -> None:
    """intersection::execute (operators/intersection/intersection.hpp:44-55)."""
    call("sg_intersection_execute", G.handle, in1.handle, in2.handle, out.handle)


intersection = _types.SimpleNamespace(execute=_intersect)


def segmented_intersection(G: Graph, a, b) -> np.ndarray:
    """|N(a[i]) n N(b[i])| for each pair (GraphCSRDevice::getIntersectionCount,
    graph/impls/graph_csr.hpp:109-135)."""
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    da, db = DeviceArray(a), DeviceArray(b)
    dc = DeviceArray(shape=a.size, dtype=np.uint32)
    call("sg_segmented_intersection", G.handle, C.cast(da.ptr, _lib.u32p), C.cast(db.ptr, _lib.u32p), a.size,
         C.cast(dc.ptr, _lib.u32p))
    return dc.numpy()
