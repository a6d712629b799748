"""sg_bfs_noalloc: the BFS entry point for callers that cannot allocate
device memory (a latency-critical loop that must not enter the CUDA
allocator, or a plug-in whose host application owns all device memory).

Its working memory is a static device array inside the library, so the
test checks that two calls in a row, sharing that array, give the same
depths as the allocating entry point (sg_run_bfs) and as the oracle's BFS;
depths are integers, so the comparison is exact.  Two graphs at the entry
point's vertex limit (2^22) fill its heavy-vertex lists (directed: 2^19
vertices of out-degree 256, the list's capacity; undirected: 2^18 hubs).
The file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(sg):
    fn = sg._lib.lib.sg_bfs_noalloc
    u32p = C.POINTER(C.c_uint32)
    fn.restype = C.c_int
    fn.argtypes = [u32p, u32p, u32p, u32p, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int, C.c_float, C.c_float, u32p,
                   C.POINTER(C.c_uint64), C.c_void_p]
    return fn


def _reference_depths(sg, G, source, direction):
    out = np.empty(G.getVertexCount(), np.uint32)
    d = sg._lib.BfsDetails()
    sg._lib.call("sg_run_bfs", G.handle, source, direction, C.c_float(15.0), C.c_float(24.0),
                 out.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(d))
    return out, int(d.iterations)


def _call(fn, sg, G, g, directed, src, direction, depth, m=None):
    fwd, inv = G.device_view(False), G.device_view(True)
    it = C.c_uint64()
    st = fn(fwd.row_offsets, fwd.column_indices, inv.row_offsets if directed else None,
            inv.column_indices if directed else None, g.n, g.m if m is None else m, src, direction, 15.0, 24.0,
            C.cast(depth.ptr, C.POINTER(C.c_uint32)), C.byref(it), None)
    return st, it.value


@pytest.mark.parametrize("directed", [False, True])
def test_noalloc_matches_allocating_bfs_twice(sg, rmat, oracle, directed):
    fn = _bind(sg)
    if directed:
        rng = np.random.default_rng(4)
        n = 20000
        g = sg.io.fromCOO(n, rng.integers(0, n, 90000), rng.integers(0, n, 90000), dedupe=True,
                          drop_self_loops=True)
        G = sg.graph.build.fromCSR(g, sg.Properties(directed=True))
    else:
        g = rmat(14, perm_seed=5)
        G = sg.graph.build.fromCSR(g)
    fwd, inv = G.device_view(False), G.device_view(True)
    n = g.n
    depth = sg.DeviceArray(shape=n, dtype=np.uint32)
    srcs = [int(np.argmax(g.degrees())), int(sg.io.sample_sources(g, 1, seed=11)[0])]
    for direction, src in zip((2, 0), srcs):  # two calls in a row share the static scratch
        it = C.c_uint64()
        st = fn(fwd.row_offsets, fwd.column_indices, inv.row_offsets if directed else None,
                inv.column_indices if directed else None, n, g.m, src, direction, 15.0, 24.0,
                C.cast(depth.ptr, C.POINTER(C.c_uint32)), C.byref(it), None)
        assert st == 0, sg._lib.lib.sg_last_error().decode()
        want, want_it = _reference_depths(sg, G, src, direction)
        assert np.array_equal(depth.numpy(), want)
        assert it.value == want_it
        assert np.array_equal(want, oracle.bfs_levels(g, src))


def _hub_tree_directed(sg):
    """n = 2^22: hubs 0..2^19-1 of out-degree exactly 256 (tree edges to hubs
    2h+1, 2h+2, the rest to leaves), leaves without out-edges; m = 2^27."""
    n, H = 1 << 22, 1 << 19
    L = n - H
    h = np.arange(H, dtype=np.int64)[:, None]
    j = np.arange(256, dtype=np.int64)[None, :]
    col = H + (h * 256 + j) % L
    for k in (0, 1):
        child = 2 * h[:, 0] + 1 + k
        col[:, k] = np.where(child < H, child, col[:, k])
    ro = np.concatenate([np.arange(H + 1, dtype=np.int64) * 256, np.full(L, H * 256, np.int64)])
    return sg.CSR(ro.astype(np.uint32), col.reshape(-1).astype(np.uint32), properties=sg.Properties(directed=True))


def _hub_tree_undirected(sg):
    """n = 2^22: 2^18 hubs linked as a binary tree, each joined to 255 leaves;
    every leaf is joined to exactly 17 hubs; m = 134,217,726."""
    n, H = 1 << 22, 1 << 18
    L = n - H
    assert H * 255 == 17 * L
    h = np.arange(H, dtype=np.int64)
    tree = np.stack([np.where(h > 0, (h - 1) // 2, -1), np.where(2 * h + 1 < H, 2 * h + 1, -1),
                     np.where(2 * h + 2 < H, 2 * h + 2, -1)], axis=1)
    leaves = H + (h[:, None] * 255 + np.arange(255, dtype=np.int64)[None, :]) % L
    hub_rows = np.concatenate([tree, leaves], axis=1)
    keep = hub_rows >= 0
    hub_deg = keep.sum(axis=1)
    r = np.arange(L, dtype=np.int64)[:, None]
    leaf_rows = (r + np.arange(17, dtype=np.int64)[None, :] * L) // 255
    deg = np.concatenate([hub_deg, np.full(L, 17, np.int64)])
    ro = np.zeros(n + 1, np.int64)
    np.cumsum(deg, out=ro[1:])
    col = np.concatenate([hub_rows[keep], leaf_rows.reshape(-1)])
    return sg.CSR(ro.astype(np.uint32), col.astype(np.uint32))


@pytest.mark.parametrize("directed", [True, False])
def test_noalloc_at_its_vertex_limit(sg, oracle, directed):
    fn = _bind(sg)
    g = _hub_tree_directed(sg) if directed else _hub_tree_undirected(sg)
    assert g.n == 1 << 22 and g.m <= 1 << 27
    assert int((g.degrees() >= 256).sum()) == (1 << 19 if directed else 1 << 18)
    G = sg.graph.build.fromCSR(g, sg.Properties(directed=directed))
    depth = sg.DeviceArray(shape=g.n, dtype=np.uint32)
    for direction, src in ((2, 0), (0, 5)):  # hybrid from the root hub, then push from another hub
        st, it = _call(fn, sg, G, g, directed, src, direction, depth)
        assert st == 0, sg._lib.lib.sg_last_error().decode()
        want, want_it = _reference_depths(sg, G, src, direction)
        got = depth.numpy()
        assert np.array_equal(got, want)
        assert it == want_it
        assert np.array_equal(got, oracle.bfs_levels(g, src))
    # an edge count that is not row_offsets[n] would undersize the heavy lists
    st, _ = _call(fn, sg, G, g, directed, 0, 2, depth, m=g.m // 2)
    assert st == sg._lib.SG_ERR_INVALID
    assert "row_offsets[n]" in sg._lib.lib.sg_last_error().decode()


def test_noalloc_rejects_graphs_over_its_limit(sg):
    fn = _bind(sg)
    dummy = (C.c_uint32 * 4)()
    p = C.cast(dummy, C.POINTER(C.c_uint32))
    st = fn(p, p, None, None, (1 << 22) + 1, 10, 0, 0, 1.0, 1.0, p, None, None)
    assert st == sg._lib.SG_ERR_INVALID
    assert "2^22" in sg._lib.lib.sg_last_error().decode()
    st = fn(p, p, None, None, 100, (1 << 27) + 1, 0, 0, 1.0, 1.0, p, None, None)
    assert st == sg._lib.SG_ERR_INVALID
    assert "2^27" in sg._lib.lib.sg_last_error().decode()
