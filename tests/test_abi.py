"""The C ABI without a GPU: the library loads, exports every entry point that
include/sygraph_b200.h declares, and the host-only calls (graph generation,
CSR conversion, binary / Matrix Market I/O, argument checks) behave."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "sygraph_b200.h"
LIB = ROOT / "sygraph_b200" / "libsygraph_b200.so"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert len(names) > 60
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (sg_[a-z0-9_]+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = C.CDLL(str(LIB))
    for n in names:
        assert getattr(lib, n) is not None


def test_python_binding_covers_the_header(sg):
    bound = set(sg._lib.SIGNATURES) | set(sg._lib.OPTIONAL)
    assert not sg._lib.MISSING
    # every entry point of the header has a ctypes signature or is bound at its call site
    unbound = [n for n in declared_symbols() if n not in bound and n != "sg_bfs_noalloc"]
    assert not unbound, unbound


def test_status_strings(sg):
    lib = sg._lib.lib
    assert lib.sg_status_string(0) == b"SG_OK"
    assert lib.sg_status_string(4) == b"SG_ERR_TIMEOUT"
    assert b"sm_100a" in lib.sg_version()


def test_rmat_generator_properties(sg):
    g = sg.io.rmat(10, perm_seed=0)
    ro, col = g.row_offsets, g.column_indices
    assert g.n == 1024 and ro[0] == 0 and ro[-1] == g.m
    for v in range(g.n):
        row = col[ro[v]:ro[v + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)  # sorted, no duplicates
        assert not np.any(row == v)  # no self-loops
    # symmetric, with symmetric weights
    w = g.values
    pairs = {}
    for v in range(g.n):
        for e in range(ro[v], ro[v + 1]):
            pairs[(v, int(col[e]))] = w[e]
    for (a, b), x in pairs.items():
        assert pairs[(b, a)] == x
    assert w.min() > 0 and w.max() <= 1.0
    assert np.array_equal(sg.io.rmat(10, perm_seed=0).column_indices, col)  # deterministic


def test_grid_generator(sg):
    g = sg.io.grid(16, 0.0, value_type=sg.WEIGHT_U32)
    assert g.n == 256 and g.m == 2 * 2 * 16 * 15
    assert g.values.min() >= 1 and g.values.max() <= 64


def test_binary_and_mm_roundtrip(sg, tmp_path, golden):
    g = sg.io.rmat(8, perm_seed=3)
    p = tmp_path / "g.bin"
    sg.io.toBinary(g, p, sg.Properties(directed=False, weighted=True))
    h = sg.io.fromBinary(p, sg.WEIGHT_F32)
    assert np.array_equal(h.row_offsets, g.row_offsets)
    assert np.array_equal(h.column_indices, g.column_indices)
    assert np.array_equal(h.values, g.values)
    assert not h.properties.directed and h.properties.weighted
    raw = p.read_bytes()
    assert int.from_bytes(raw[:8], "little") == golden["binary_csr"]["magic"]
    # legacy headerless layout: rows, nnz, arrays
    legacy = tmp_path / "legacy.bin"
    legacy.write_bytes(raw[16:])
    h2 = sg.io.fromBinary(legacy, sg.WEIGHT_F32)
    assert np.array_equal(h2.column_indices, g.column_indices) and h2.properties.directed
    mm = tmp_path / "m.mtx"
    mm.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n4 4 3\n2 1\n3 2\n4 3\n")
    m = sg.io.fromMM(mm, sg.WEIGHT_U32)
    assert m.row_offsets.tolist() == [0, 1, 3, 5, 6]
    assert m.column_indices.tolist() == [1, 0, 2, 1, 3, 2]
    assert not m.properties.directed and not m.properties.weighted


def test_csr_invert_and_coo(sg):
    g = sg.io.fromCOO(4, [0, 0, 1, 3], [1, 2, 2, 0], values=np.array([1, 2, 3, 4], np.uint32))
    inv = g.invert()
    assert inv.row_offsets.tolist() == [0, 1, 2, 4, 4]
    assert inv.column_indices.tolist() == [3, 0, 0, 1]
    assert inv.values.tolist() == [4, 1, 2, 3]


def test_argument_errors_without_gpu(sg):
    lib = sg._lib.lib
    out = C.c_void_p()
    ro = np.array([0, 2], np.uint32)  # last offset != m
    st = lib.sg_graph_create_csr(ro.ctypes.data_as(C.POINTER(C.c_uint32)), None, None, 0, 1, 0, 0, None,
                                 C.byref(out))
    assert st == sg._lib.SG_ERR_INVALID
    assert lib.sg_msbfs_create(None, 64, C.byref(out)) == sg._lib.SG_ERR_INVALID
    with pytest.raises(sg._lib.SygraphError):
        sg.io.rmat(0)


def _create(sg, ro, col, flags):
    lib = sg._lib.lib
    out = C.c_void_p()
    ro = np.ascontiguousarray(ro, np.uint32)
    col = np.ascontiguousarray(col, np.uint32)
    st = lib.sg_graph_create_csr(ro.ctypes.data_as(C.POINTER(C.c_uint32)), col.ctypes.data_as(C.POINTER(C.c_uint32)),
                                 None, 0, ro.size - 1, col.size, flags, None, C.byref(out))
    return st, out


@pytest.mark.parametrize("flags", [0, 1])  # undirected, directed
def test_malformed_csr_is_rejected_before_upload(sg, flags):
    """A column index >= n or decreasing offsets would make every kernel index
    outside its per-vertex arrays: the graph is refused on the host."""
    st, out = _create(sg, [0, 2, 3, 4], [1, 7, 0, 0], flags)  # column 7 with n = 3
    assert st == sg._lib.SG_ERR_INVALID and not out.value
    assert b"column index out of range at edge 1" in sg._lib.lib.sg_last_error()
    st, out = _create(sg, [0, 3, 1, 4], [1, 2, 0, 1], flags)  # offsets 3 -> 1
    assert st == sg._lib.SG_ERR_INVALID and not out.value
    assert b"row_offsets decrease at row 1" in sg._lib.lib.sg_last_error()


def test_malformed_binary_csr_is_rejected(sg, tmp_path):
    g = sg.io.rmat(6, perm_seed=3)
    good = tmp_path / "g.bin"
    sg.io.toBinary(g, good)
    raw = bytearray(good.read_bytes())
    body = 32 + 4 * (g.n + 1)  # 32-byte header, then row offsets, then columns
    bad_col = bytearray(raw)
    bad_col[body:body + 4] = (g.n + 5).to_bytes(4, "little")
    (tmp_path / "c.bin").write_bytes(bad_col)
    with pytest.raises(sg._lib.SygraphError, match="column index out of range"):
        sg.io.fromBinary(tmp_path / "c.bin")
    bad_ro = bytearray(raw)
    bad_ro[32 + 4 * 2:32 + 4 * 3] = (g.m).to_bytes(4, "little")  # row 1 ends at m, row 2 ends lower
    (tmp_path / "r.bin").write_bytes(bad_ro)
    with pytest.raises(sg._lib.SygraphError, match="row_offsets decrease"):
        sg.io.fromBinary(tmp_path / "r.bin")
