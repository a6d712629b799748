"""Host-side objects over the C ABI: CSR containers, device graphs, frontiers
and device arrays.  Names follow the reference (formats::CSR,
graph::build::fromCSR, frontier::makeFrontier, Frontier methods)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call, lib

WEIGHT_NONE, WEIGHT_F32, WEIGHT_U32 = 0, 1, 2
GRAPH_DIRECTED, GRAPH_WEIGHTED = 1, 2

_NP_OF_WT = {WEIGHT_F32: np.float32, WEIGHT_U32: np.uint32}


def _ptr(a: np.ndarray | None, ctype=C.c_uint32):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _vptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


@dataclass
class Properties:
    """graph::Properties (graph/properties.hpp:29-32)."""
    directed: bool = False
    weighted: bool = False

    @property
    def flags(self) -> int:
        return (GRAPH_DIRECTED if self.directed else 0) | (GRAPH_WEIGHTED if self.weighted else 0)


class CSR:
    """formats::CSR (formats/csr.hpp:32-215): uint32 row offsets and column
    indices, float32 or uint32 values (or none)."""

    def __init__(self, row_offsets, column_indices, values=None, value_type: int | None = None,
                 properties: Properties | None = None):
        self.row_offsets = np.ascontiguousarray(row_offsets, dtype=np.uint32)
        self.column_indices = np.ascontiguousarray(column_indices, dtype=np.uint32)
        if values is not None:
            values = np.asarray(values)
            if value_type is None:
                value_type = WEIGHT_F32 if values.dtype.kind == "f" else WEIGHT_U32
            values = np.ascontiguousarray(values, dtype=_NP_OF_WT[value_type])
        self.values = values
        self.value_type = WEIGHT_NONE if values is None else value_type
        self.properties = properties or Properties(weighted=values is not None)
        if self.row_offsets.size < 1 or self.row_offsets[0] != 0 or self.row_offsets[-1] != self.column_indices.size:
            raise ValueError("row_offsets must start at 0 and end at the number of column indices")

    @property
    def n(self) -> int:
        return int(self.row_offsets.size - 1)

    @property
    def m(self) -> int:
        return int(self.column_indices.size)

    def getRowOffsetsSize(self) -> int:
        return self.n

    def getNumNonzeros(self) -> int:
        return self.m

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_offsets.astype(np.int64)).astype(np.uint32)

    # ---- conversions through the C ABI
    def _to_host(self) -> _lib.HostCSR:
        h = _lib.HostCSR()
        h.n = self.n
        h.m = self.m
        h.row_offsets = _ptr(self.row_offsets)
        h.column_indices = _ptr(self.column_indices)
        h.values = _vptr(self.values)
        h.value_type = self.value_type
        h.flags = self.properties.flags
        return h

    @staticmethod
    def _from_host(h: _lib.HostCSR, free: bool = True) -> "CSR":
        n, m = int(h.n), int(h.m)
        ro = np.ctypeslib.as_array(h.row_offsets, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(h.column_indices, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        vals = None
        if h.values and h.value_type != WEIGHT_NONE:
            raw = np.ctypeslib.as_array(C.cast(h.values, C.POINTER(C.c_uint32)), shape=(m,)).copy() if m else \
                np.zeros(0, np.uint32)
            vals = raw.view(_NP_OF_WT[h.value_type])
        props = Properties(directed=bool(h.flags & GRAPH_DIRECTED), weighted=bool(h.flags & GRAPH_WEIGHTED))
        out = CSR(ro, col, vals, h.value_type if vals is not None else None, props)
        if free:
            lib.sg_host_csr_free(C.byref(h))
        return out

    def invert(self) -> "CSR":
        """formats::CSR::invert (formats/csr.hpp:179-209)."""
        h_in = self._to_host()
        h_out = _lib.HostCSR()
        call("sg_csr_invert", C.byref(h_in), C.byref(h_out))
        return CSR._from_host(h_out)


class DeviceArray:
    """A device buffer with numpy round trips (plain cudaMalloc through the C ABI)."""

    def __init__(self, data: np.ndarray | None = None, *, shape=None, dtype=None, stream=None):
        if data is not None:
            data = np.ascontiguousarray(data)
            shape, dtype = data.shape, data.dtype
        self.shape = tuple(np.atleast_1d(shape)) if shape is not None else (0,)
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        self.stream = stream
        p = C.c_void_p()
        call("sg_malloc_device", max(self.nbytes, 1), C.byref(p))
        self.ptr = p.value
        if data is not None:
            call("sg_memcpy", C.c_void_p(self.ptr), C.c_void_p(data.ctypes.data), self.nbytes, 0, stream)
        else:
            call("sg_memset", C.c_void_p(self.ptr), 0, self.nbytes, stream)

    def numpy(self) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        call("sg_memcpy", C.c_void_p(out.ctypes.data), C.c_void_p(self.ptr), self.nbytes, 1, self.stream)
        return out

    def upload(self, data: np.ndarray) -> None:
        data = np.ascontiguousarray(data, dtype=self.dtype)
        assert data.nbytes == self.nbytes
        call("sg_memcpy", C.c_void_p(self.ptr), C.c_void_p(data.ctypes.data), self.nbytes, 0, self.stream)

    def fill(self, value) -> None:
        self.upload(np.full(self.shape, value, self.dtype))

    def __del__(self):
        p = getattr(self, "ptr", None)
        if p and lib is not None:
            lib.sg_free_device(C.c_void_p(p))
            self.ptr = None


class Graph:
    """graph::detail::GraphCSR (graph/impls/graph_csr.hpp:158-439): owns the
    device CSR (and the inverse CSR of a directed graph)."""

    def __init__(self, csr: CSR, properties: Properties | None = None, stream=None):
        props = properties or csr.properties
        h = C.c_void_p()
        call("sg_graph_create_csr", _ptr(csr.row_offsets), _ptr(csr.column_indices), _vptr(csr.values),
             csr.value_type, csr.n, csr.m, props.flags, stream, C.byref(h))
        self._adopt(h, stream, csr)

    def _adopt(self, h, stream, csr: CSR | None) -> None:
        self.handle = h
        self.stream = stream
        self._csr = csr
        n, m, flags, vt = C.c_uint32(), C.c_uint64(), C.c_uint32(), C.c_int()
        call("sg_graph_info", h, C.byref(n), C.byref(m), C.byref(flags), C.byref(vt))
        self._n, self._m, self.value_type = n.value, m.value, vt.value
        self.properties = Properties(directed=bool(flags.value & GRAPH_DIRECTED),
                                     weighted=bool(flags.value & GRAPH_WEIGHTED))
        if csr is not None:
            self.properties = csr.properties if csr.properties.flags == flags.value else self.properties

    @classmethod
    def from_handle(cls, h, stream=None) -> "Graph":
        """Wraps a graph the library built on the device; its host CSR is
        copied back only when asked for (`csr`)."""
        g = cls.__new__(cls)
        g._adopt(h, stream, None)
        return g

    @property
    def csr(self) -> CSR:
        if self._csr is None:
            ro = np.empty(self._n + 1, np.uint32)
            col = np.empty(self._m, np.uint32)
            val = np.empty(self._m, _NP_OF_WT[self.value_type])
            call("sg_graph_copy_csr", self.handle, 0, _ptr(ro), _ptr(col), C.c_void_p(val.ctypes.data))
            weighted = self.properties.weighted
            self._csr = CSR(ro, col, val if weighted else None, self.value_type if weighted else None,
                            self.properties)
        return self._csr

    def getVertexCount(self) -> int:
        return self._n

    def getEdgeCount(self) -> int:
        return self._m

    def getDegree(self, v: int) -> int:
        return int(self.csr.row_offsets[v + 1] - self.csr.row_offsets[v])

    def getRowOffsets(self) -> np.ndarray:
        return self.csr.row_offsets

    def getColumnIndices(self) -> np.ndarray:
        return self.csr.column_indices

    def getValues(self):
        return self.csr.values

    def device_view(self, inverse: bool = False) -> _lib.GraphView:
        v = _lib.GraphView()
        call("sg_graph_device_view", self.handle, int(inverse), C.byref(v))
        return v

    def memory_bytes(self) -> int:
        b = C.c_uint64()
        call("sg_graph_memory_bytes", self.handle, C.byref(b))
        return b.value

    def weight_sorted(self):
        """(columns, values, symmetric): the forward rows sorted by weight, as
        delta-stepping SSSP reads them (sg_graph_weight_sorted)."""
        m = self.getEdgeCount()
        col = np.empty(m, np.uint32)
        val = np.empty(m, _NP_OF_WT[self.value_type])
        sym = C.c_int()
        call("sg_graph_weight_sorted", self.handle, _ptr(col), C.c_void_p(val.ctypes.data), C.byref(sym))
        return col, val, bool(sym.value)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_graph_destroy(h)
            self.handle = None


class build:  # noqa: N801 - mirrors graph::build
    @staticmethod
    def fromCSR(csr: CSR, properties: Properties | None = None, stream=None) -> Graph:
        """graph::build::fromCSR (graph/build.hpp:31-41)."""
        return Graph(csr, properties, stream)

    @staticmethod
    def fromCOO(n: int, src, dst, values=None, value_type: int | None = None, symmetrize: bool = False,
                dedupe: bool = False, drop_self_loops: bool = False, stream=None) -> Graph:
        """Edge list -> device graph, built on the device (sg_graph_create_coo):
        the same CSR as io.fromCOO + fromCSR.  src / dst / values are host
        arrays, or DeviceArray objects already on the device."""
        dev = isinstance(src, DeviceArray)
        if dev:
            count = int(np.prod(src.shape))
            ps, pd = C.c_void_p(src.ptr), C.c_void_p(dst.ptr)
            pv = C.c_void_p(values.ptr) if values is not None else None
            if value_type is None:
                value_type = WEIGHT_NONE if values is None else (WEIGHT_F32 if values.dtype == np.float32
                                                                 else WEIGHT_U32)
            keep = ()
        else:
            s_ = np.ascontiguousarray(src, np.uint32)
            d_ = np.ascontiguousarray(dst, np.uint32)
            if s_.size != d_.size:
                raise ValueError("src and dst must have the same length")
            count = s_.size
            v_ = None
            if values is not None:
                values = np.asarray(values)
                if value_type is None:
                    value_type = WEIGHT_F32 if values.dtype.kind == "f" else WEIGHT_U32
                v_ = np.ascontiguousarray(values, _NP_OF_WT[value_type])
            elif value_type is None:
                value_type = WEIGHT_NONE
            ps, pd = C.c_void_p(s_.ctypes.data), C.c_void_p(d_.ctypes.data)
            pv = None if v_ is None else C.c_void_p(v_.ctypes.data)
            keep = (s_, d_, v_)
        h = C.c_void_p()
        call("sg_graph_create_coo", ps, pd, pv, value_type, int(n), int(count), int(symmetrize), int(dedupe),
             int(drop_self_loops), int(dev), stream, C.byref(h))
        del keep
        return Graph.from_handle(h, stream)


class Frontier:
    """Frontier<T, frontier_type::mlb> (frontier/impls/mlb_frontier.hpp:155-449)."""

    def __init__(self, num_elems: int, stream=None):
        h = C.c_void_p()
        call("sg_frontier_create", num_elems, stream, C.byref(h))
        self.handle = h
        self.num_elems = num_elems

    def getNumElems(self) -> int:
        return self.num_elems

    def insert(self, idx: int) -> bool:
        call("sg_frontier_insert", self.handle, idx)
        return True

    def insert_list(self, ids) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        call("sg_frontier_insert_list", self.handle, _ptr(ids), ids.size)

    def remove(self, idx: int) -> bool:
        call("sg_frontier_remove", self.handle, idx)
        return True

    def check(self, idx: int) -> bool:
        r = C.c_int()
        call("sg_frontier_check", self.handle, idx, C.byref(r))
        return bool(r.value)

    def empty(self) -> bool:
        r = C.c_int()
        call("sg_frontier_empty", self.handle, C.byref(r))
        return bool(r.value)

    def size(self) -> int:
        r = C.c_uint64()
        call("sg_frontier_size", self.handle, C.byref(r))
        return r.value

    def clear(self) -> None:
        call("sg_frontier_clear", self.handle)

    def merge(self, other: "Frontier") -> None:
        call("sg_frontier_merge", self.handle, other.handle)

    def intersect(self, other: "Frontier") -> None:
        call("sg_frontier_intersect", self.handle, other.handle)

    def computeActiveFrontier(self, invert: bool = False) -> int:
        r = C.c_uint32()
        call("sg_frontier_compact", self.handle, int(invert), C.byref(r))
        return r.value

    def saveState(self):
        v = self.device_view()
        l0 = np.zeros(v.words0, np.uint32)
        l1 = np.zeros(v.words1, np.uint32)
        call("sg_frontier_save", self.handle, _ptr(l0), _ptr(l1))
        return (l0, l1)

    def loadState(self, state) -> None:
        l0, l1 = state
        call("sg_frontier_load", self.handle, _ptr(l0), _ptr(l1))

    def flags(self) -> np.ndarray:
        out = np.zeros(self.num_elems, np.uint8)
        call("sg_frontier_to_flags", self.handle, _ptr(out, C.c_uint8))
        return out

    def active(self) -> list[int]:
        return [int(i) for i in np.nonzero(self.flags())[0]]

    def device_view(self) -> _lib.FrontierView:
        v = _lib.FrontierView()
        call("sg_frontier_device_view", self.handle, C.byref(v))
        return v

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_frontier_destroy(h)
            self.handle = None


def makeFrontier(graph: Graph, view: str = "vertex") -> Frontier:
    """frontier::makeFrontier<View, Type> (frontier/frontier.hpp:68-80)."""
    if view == "vertex":
        return Frontier(graph.getVertexCount(), graph.stream)
    if view == "edge":
        return Frontier(graph.getEdgeCount(), graph.stream)
    raise ValueError("Invalid frontier view")


def swap(a: Frontier, b: Frontier) -> None:
    """frontier::swap (frontier/frontier.hpp:94-101)."""
    call("sg_frontier_swap", a.handle, b.handle)


def launch_count() -> int:
    return int(lib.sg_kernel_launch_count())


def device_count() -> int:
    c = C.c_int()
    st = lib.sg_device_count(C.byref(c))
    return c.value if st == 0 else 0
