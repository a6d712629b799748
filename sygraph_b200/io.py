"""Graph inputs: io::csr readers and writers (io/read_csr.hpp), the dense
adjacency-matrix text format of the reference fixtures
(io::csr::fromMatrix, io/read_csr.hpp:40-67) and the seeded generators."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call
from .core import CSR, WEIGHT_F32, WEIGHT_NONE, WEIGHT_U32, Properties, _ptr, _vptr


def fromMatrix(text: str, value_type: int = WEIGHT_U32, properties: Properties | None = None) -> CSR:
    """io::csr::fromMatrix: first token n, then an n x n matrix; every non-zero
    entry (row i, column j) becomes an edge i -> j with that value."""
    toks = text.split()
    n = int(toks[0])
    vals = np.array([float(t) for t in toks[1:1 + n * n]], dtype=np.float64).reshape(n, n)
    rows, cols = np.nonzero(vals)
    ro = np.zeros(n + 1, np.uint32)
    np.add.at(ro, rows + 1, 1)
    ro = np.cumsum(ro, dtype=np.uint64).astype(np.uint32)
    dt = np.float32 if value_type == WEIGHT_F32 else np.uint32
    return CSR(ro, cols.astype(np.uint32), vals[rows, cols].astype(dt), value_type, properties or Properties())


def fromCOO(n: int, src, dst, values=None, value_type: int | None = None, symmetrize: bool = False,
            dedupe: bool = False, drop_self_loops: bool = False) -> CSR:
    """io::csr::fromCOO (io/read_csr.hpp:260-300), with optional symmetrise /
    de-duplicate / self-loop removal."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    vt = WEIGHT_NONE
    vbits = None
    if values is not None:
        values = np.asarray(values)
        vt = value_type or (WEIGHT_F32 if values.dtype.kind == "f" else WEIGHT_U32)
        vbits = np.ascontiguousarray(values, dtype=np.float32 if vt == WEIGHT_F32 else np.uint32)
    h = _lib.HostCSR()
    call("sg_csr_from_edges", n, _ptr(src), _ptr(dst), _vptr(vbits), vt, src.size, int(symmetrize), int(dedupe),
         int(drop_self_loops), C.byref(h))
    return CSR._from_host(h)


def fromBinary(path: str, value_type: int = WEIGHT_F32) -> CSR:
    """io::csr::fromBinary (io/read_csr.hpp:365-411), including the legacy
    headerless layout."""
    h = _lib.HostCSR()
    call("sg_csr_read_binary", str(path).encode(), value_type, C.byref(h))
    return CSR._from_host(h)


def toBinary(csr: CSR, path: str, properties: Properties | None = None) -> None:
    """io::csr::toBinary (io/read_csr.hpp:316-349)."""
    h = csr._to_host()
    if properties is not None:
        h.flags = properties.flags
    call("sg_csr_write_binary", C.byref(h), str(path).encode())


def fromMM(path: str, value_type: int = WEIGHT_F32) -> CSR:
    """io::csr::fromMM (io/read_csr.hpp:88-192)."""
    h = _lib.HostCSR()
    call("sg_csr_read_mm", str(path).encode(), value_type, C.byref(h))
    return CSR._from_host(h)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
         weight_seed: int = 2, perm_seed: int = 0, value_type: int = WEIGHT_F32) -> CSR:
    """Seeded RMAT graph: symmetrised, self-loops and duplicates removed,
    sorted adjacency; weights keyed by the unordered pair (float32 on (0,1]
    or uint32 on [1,64])."""
    p = _lib.RmatParams(scale, edge_factor, a, b, c, seed, weight_seed, perm_seed, value_type)
    h = _lib.HostCSR()
    call("sg_rmat_generate", C.byref(p), C.byref(h))
    return CSR._from_host(h)


def grid(side: int, long_range_frac: float = 0.02, seed: int = 1, weight_seed: int = 2,
         value_type: int = WEIGHT_U32) -> CSR:
    """side x side 4-neighbour grid plus uniform random long-range pairs."""
    h = _lib.HostCSR()
    call("sg_grid_generate", side, long_range_frac, seed, weight_seed, value_type, C.byref(h))
    return CSR._from_host(h)


def sample_sources(csr: CSR, k: int, seed: int = 3) -> np.ndarray:
    """k distinct vertices with degree > 0, drawn uniformly with `seed`."""
    out = np.zeros(k, np.uint32)
    h = csr._to_host()
    call("sg_sample_sources", C.byref(h), k, seed, _ptr(out))
    return out


def max_degree_vertex(csr: CSR) -> int:
    """Vertex of maximum degree, lowest id on ties."""
    return int(np.argmax(csr.degrees()))
