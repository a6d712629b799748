"""The oracle: a CPU restatement of SYgraph's frontier algorithms.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
CPU-baseline / reference leg of bench.py may import this package, and only as
the checker or the timed CPU baseline; the product (sygraph_b200) never calls
it.  The C code is oracle/sg_oracle.c, built into oracle/libsg_oracle.so by
oracle/Makefile (gcc -O3 -fopenmp).

Parity pinning: the reference (SYCL) cannot be compiled without a SYCL
compiler, so these functions are pinned against the reference's own
known-answer fixtures and assertions, committed under tests/golden/ by
tests/golden/make_golden.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libsg_oracle.so"


def build(force: bool = False) -> Path:
    src = HERE / "sg_oracle.c"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)] + (["-B"] if force else []), check=True)
    return LIB


def _load() -> C.CDLL:
    build()
    lib = C.CDLL(str(LIB))
    u32p, u8p, u64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint8), C.POINTER(C.c_uint64)
    f32p, f64p = C.POINTER(C.c_float), C.POINTER(C.c_double)
    sig = {
        "or_bfs_levels": (None, [C.c_uint32, u32p, u32p, C.c_uint32, u32p]),
        "or_bfs_frontier": (C.c_int64, [C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32, C.c_int, C.c_float,
                                        C.c_float, u32p, u8p, C.c_uint64, C.c_int]),
        "or_sssp_dijkstra_f32": (None, [C.c_uint32, u32p, u32p, f32p, C.c_uint32, f32p]),
        "or_sssp_dijkstra_u32": (None, [C.c_uint32, u32p, u32p, u32p, C.c_uint32, u32p]),
        "or_sssp_frontier_f32": (C.c_int64, [C.c_uint32, u32p, u32p, f32p, C.c_uint32, f32p, C.c_int]),
        "or_cc_maxlabel": (None, [C.c_uint32, u32p, u32p, u32p]),
        "or_bc": (None, [C.c_uint32, u32p, u32p, u32p, C.c_uint32, f64p, C.c_int]),
        "or_tc_edge_merge": (C.c_uint64, [C.c_uint32, u32p, u32p, u64p, C.c_int]),
        "or_tc_dag": (C.c_uint64, [C.c_uint32, u32p, u32p, u64p, C.c_int]),
        "or_bfs_multi": (None, [C.c_uint32, u32p, u32p, u32p, C.c_uint32, u32p, C.c_int]),
        "or_visited_edges": (C.c_uint64, [C.c_uint32, u32p, u32p, C.c_uint32]),
        "or_rmat_generate": (C.c_int64, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                         C.c_uint64, C.c_uint64, C.c_int, C.POINTER(u32p), C.POINTER(u32p),
                                         C.POINTER(u32p)]),
        "or_sample_sources": (C.c_int, [C.c_uint32, u32p, C.c_uint32, C.c_uint64, u32p]),
        "or_free": (None, [C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()


def _p(a, t=C.c_uint32):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _csr(csr):
    ro = np.ascontiguousarray(csr.row_offsets, np.uint32)
    col = np.ascontiguousarray(csr.column_indices, np.uint32)
    return int(ro.size - 1), ro, col


def threads() -> int:
    return os.cpu_count() or 1


def bfs_levels(csr, source: int) -> np.ndarray:
    """examples/bfs/bfs.cpp:16-56 (serial level-synchronous)."""
    n, ro, col = _csr(csr)
    out = np.empty(n, np.uint32)
    _lib.or_bfs_levels(n, _p(ro), _p(col), source, _p(out))
    return out


def bfs_frontier(csr, source: int, direction: int = 0, alpha: float = 1.0, beta: float = 1.0, inverse=None,
                 nthreads: int = 0):
    """algorithms/bfs.hpp:153-350 restated; returns (depth, iterations, step_is_pull list)."""
    n, ro, col = _csr(csr)
    if inverse is None:
        iro, icol = ro, col
    else:
        _, iro, icol = _csr(inverse)
    depth = np.empty(n, np.uint32)
    cap = n + 2
    steps = np.zeros(cap, np.uint8)
    it = _lib.or_bfs_frontier(n, _p(ro), _p(col), _p(iro), _p(icol), source, direction, alpha, beta, _p(depth),
                              _p(steps, C.c_uint8), cap, nthreads)
    return depth, int(it), [int(x) for x in steps[:it]]


def sssp_dijkstra(csr, source: int) -> np.ndarray:
    """examples/sssp/sssp.cpp:23-66 (fp32 or uint32 by the CSR's value type)."""
    n, ro, col = _csr(csr)
    vals = csr.values
    if vals.dtype == np.float32:
        out = np.empty(n, np.float32)
        _lib.or_sssp_dijkstra_f32(n, _p(ro), _p(col), _p(vals, C.c_float), source, _p(out, C.c_float))
    else:
        out = np.empty(n, np.uint32)
        _lib.or_sssp_dijkstra_u32(n, _p(ro), _p(col), _p(np.ascontiguousarray(vals, np.uint32)), source, _p(out))
    return out


def sssp_frontier(csr, source: int, nthreads: int = 0):
    """algorithms/sssp.hpp:152-210 restated (OpenMP); returns (dist, iterations)."""
    n, ro, col = _csr(csr)
    out = np.empty(n, np.float32)
    it = _lib.or_sssp_frontier_f32(n, _p(ro), _p(col), _p(csr.values, C.c_float), source, _p(out, C.c_float),
                                   nthreads)
    return out, int(it)


def cc_maxlabel(csr) -> np.ndarray:
    """algorithms/cc.hpp:103-169 fixed point."""
    n, ro, col = _csr(csr)
    out = np.empty(n, np.uint32)
    _lib.or_cc_maxlabel(n, _p(ro), _p(col), _p(out))
    return out


def bc(csr, sources, nthreads: int = 0) -> np.ndarray:
    """algorithms/bc.hpp:118-200 in FP64, summed over sources."""
    n, ro, col = _csr(csr)
    s = np.ascontiguousarray(sources, np.uint32)
    out = np.empty(n, np.float64)
    _lib.or_bc(n, _p(ro), _p(col), _p(s), s.size, _p(out, C.c_double), nthreads)
    return out


def tc_edge_merge(csr, nthreads: int = 0):
    """algorithms/tc.hpp:80-138 (corrected); returns (total, per_vertex)."""
    n, ro, col = _csr(csr)
    pv = np.zeros(n, np.uint64)
    tot = _lib.or_tc_edge_merge(n, _p(ro), _p(col), _p(pv, C.c_uint64), nthreads)
    return int(tot), pv


def tc_dag(csr, per_vertex: bool = False, nthreads: int = 0):
    """Exact count on the degree-ordered DAG; returns (total, per_vertex or None)."""
    n, ro, col = _csr(csr)
    pv = np.zeros(n, np.uint64) if per_vertex else None
    tot = _lib.or_tc_dag(n, _p(ro), _p(col), _p(pv, C.c_uint64), nthreads)
    return int(tot), pv


def bfs_multi(csr, sources, nthreads: int = 0) -> np.ndarray:
    n, ro, col = _csr(csr)
    s = np.ascontiguousarray(sources, np.uint32)
    out = np.empty((s.size, n), np.uint32)
    _lib.or_bfs_multi(n, _p(ro), _p(col), _p(s), s.size, _p(out), nthreads)
    return out


def visited_edges(csr, depth, unreached: int) -> int:
    """algorithms/bfs.hpp:88-99."""
    n, ro, _ = _csr(csr)
    d = np.ascontiguousarray(depth, np.uint32)
    return int(_lib.or_visited_edges(n, _p(ro), _p(d), unreached))


class Csr:
    """A host CSR of the oracle's own (uint32 offsets and columns, uint32 or
    float32 values), so that the CPU baseline needs nothing of the product."""

    def __init__(self, row_offsets, column_indices, values=None):
        self.row_offsets = row_offsets
        self.column_indices = column_indices
        self.values = values

    @property
    def n(self) -> int:
        return int(self.row_offsets.size - 1)

    @property
    def m(self) -> int:
        return int(self.column_indices.size)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
         weight_seed: int = 2, perm_seed: int = 0, value_type: int = 1) -> Csr:
    """The benchmarks' seeded RMAT graph (value_type 0 none, 1 float32 on
    (0,1], 2 uint32 on [1,64]); the same CSR as sygraph_b200.io.rmat."""
    u32p = C.POINTER(C.c_uint32)
    ro, col, val = u32p(), u32p(), u32p()
    m = _lib.or_rmat_generate(scale, edge_factor, a, b, c, seed, weight_seed, perm_seed, value_type, C.byref(ro),
                              C.byref(col), C.byref(val))
    if m < 0:
        raise ValueError("or_rmat_generate failed")
    n = 1 << scale
    try:
        out_ro = np.ctypeslib.as_array(ro, shape=(n + 1,)).copy()
        out_col = np.ctypeslib.as_array(col, shape=(max(m, 1),))[:m].copy()
        out_val = None
        if value_type:
            out_val = np.ctypeslib.as_array(val, shape=(max(m, 1),))[:m].copy()
            if value_type == 1:
                out_val = out_val.view(np.float32)
    finally:
        for p in (ro, col, val):
            if p:
                _lib.or_free(C.cast(p, C.c_void_p))
    return Csr(out_ro, out_col, out_val)


def sample_sources(csr, k: int, seed: int = 3) -> np.ndarray:
    """k distinct vertices with degree > 0 (the benchmarks' source draw; the
    same vertices as sygraph_b200.io.sample_sources)."""
    n, ro, _ = _csr(csr)
    out = np.zeros(k, np.uint32)
    if _lib.or_sample_sources(n, _p(ro), k, seed, _p(out)) != 0:
        raise ValueError("fewer vertices with edges than requested sources")
    return out
