"""Graph construction on the device (sg_graph_create_coo) against the host
path (io.fromCOO = sg_csr_from_edges, then graph.build.fromCSR): the same row
offsets, columns, values and flags bit for bit, inverse CSR included, for
every combination of symmetrise / de-duplicate / self-loop dropping, every
weight type, edge cases and an RMAT edge list."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host(sg, n, s, d, w, sym, dd, dsl):
    return sg.io.fromCOO(n, s, d, w, symmetrize=sym, dedupe=dd, drop_self_loops=dsl)


def _same(sg, G, csr, directed):
    assert G.getVertexCount() == csr.n and G.getEdgeCount() == csr.m
    dc = G.csr
    assert np.array_equal(dc.row_offsets, csr.row_offsets)
    assert np.array_equal(dc.column_indices, csr.column_indices)
    if csr.values is not None:
        assert np.array_equal(dc.values.view(np.uint32), csr.values.view(np.uint32))
    assert G.properties.directed == directed
    if directed:  # the inverse CSR, against the host build's
        H = sg.graph.build.fromCSR(csr, sg.Properties(directed=True, weighted=csr.values is not None))
        import ctypes as C
        for inv in (1,):
            a = [np.empty(csr.n + 1, np.uint32), np.empty(csr.m, np.uint32), np.empty(csr.m, np.uint32)]
            b = [np.empty(csr.n + 1, np.uint32), np.empty(csr.m, np.uint32), np.empty(csr.m, np.uint32)]
            u32p = C.POINTER(C.c_uint32)
            for g_, x in ((G, a), (H, b)):
                sg._lib.call("sg_graph_copy_csr", g_.handle, inv, x[0].ctypes.data_as(u32p), x[1].ctypes.data_as(u32p),
                             C.c_void_p(x[2].ctypes.data))
            for x, y in zip(a, b):
                assert np.array_equal(x, y)


@pytest.mark.parametrize("sym,dd,dsl", list(itertools.product([0, 1], repeat=3)))
@pytest.mark.parametrize("wt", ["none", "f32", "u32"])
def test_matches_host_builder(sg, sym, dd, dsl, wt):
    rng = np.random.default_rng(7 + 4 * sym + 2 * dd + dsl)
    n, k = 1000, 6000
    s = rng.integers(0, n, k).astype(np.uint32)
    d = rng.integers(0, n, k).astype(np.uint32)
    s[:300] = d[:300]  # self-loops
    s[300:900] = s[900:1500]  # repeated pairs
    d[300:900] = d[900:1500]
    w = None
    if wt == "f32":
        w = (rng.integers(1, 1 << 24, k) / float(1 << 24)).astype(np.float32)
    elif wt == "u32":
        w = rng.integers(1, 65, k).astype(np.uint32)
    G = sg.graph.build.fromCOO(n, s, d, w, symmetrize=bool(sym), dedupe=bool(dd), drop_self_loops=bool(dsl))
    _same(sg, G, _host(sg, n, s, d, w, sym, dd, dsl), directed=not sym)


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 255, 256, 257, 1 << 12, (1 << 12) - 1, 100_003])
def test_sizes_around_key_bit_boundaries(sg, n):
    rng = np.random.default_rng(n)
    k = 3 * n + 5
    s = rng.integers(0, n, k).astype(np.uint32)
    d = rng.integers(0, n, k).astype(np.uint32)
    w = rng.integers(1, 1000, k).astype(np.uint32)
    for sym in (0, 1):
        G = sg.graph.build.fromCOO(n, s, d, w, symmetrize=bool(sym), dedupe=True, drop_self_loops=True)
        _same(sg, G, _host(sg, n, s, d, w, sym, 1, 1), directed=not sym)


def test_empty_and_degenerate_inputs(sg):
    e = np.zeros(0, np.uint32)
    G = sg.graph.build.fromCOO(10, e, e, symmetrize=True, dedupe=True)
    assert G.getEdgeCount() == 0 and np.array_equal(G.csr.row_offsets, np.zeros(11, np.uint32))
    loops = np.arange(5, dtype=np.uint32)
    G = sg.graph.build.fromCOO(5, loops, loops, drop_self_loops=True)
    assert G.getEdgeCount() == 0
    G = sg.graph.build.fromCOO(5, loops, loops, symmetrize=True)  # kept once, no reverse
    _same(sg, G, _host(sg, 5, loops, loops, None, 1, 0, 0), directed=False)
    with pytest.raises(sg._lib.SygraphError):
        sg.graph.build.fromCOO(5, np.array([1, 7], np.uint32), np.array([2, 3], np.uint32))


def test_rmat_edge_list_device_pointers_and_bfs(sg, oracle, rmat):
    g = rmat(16, perm_seed=4)
    ro, col = g.row_offsets, g.column_indices
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(ro))
    keep = src < col  # one direction of each pair, shuffled
    rng = np.random.default_rng(5)
    order = rng.permutation(int(keep.sum()))
    s, d, w = src[keep][order], col[keep][order], g.values[keep][order]
    ds, dd_, dw = sg.DeviceArray(s), sg.DeviceArray(d), sg.DeviceArray(w)
    G = sg.graph.build.fromCOO(g.n, ds, dd_, dw, symmetrize=True, dedupe=True, drop_self_loops=True)
    assert np.array_equal(G.csr.row_offsets, ro) and np.array_equal(G.csr.column_indices, col)
    assert np.array_equal(G.csr.values.view(np.uint32), g.values.view(np.uint32))
    b = sg.algorithms.BFS(G)
    src0 = int(np.argmax(g.degrees()))
    b.init(src0)
    b.run(sg.algorithms.bfs_direction.hybrid, 15.0, 24.0)
    assert np.array_equal(b.getDistances(), oracle.bfs_levels(g, src0))
