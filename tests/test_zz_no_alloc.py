"""sg_bfs_noalloc: the BFS entry point for callers that cannot allocate
device memory (a latency-critical loop that must not enter the CUDA
allocator, or a plug-in whose host application owns all device memory).

Its working memory is a static device array inside the library, so the
test checks that two calls in a row, sharing that array, give the same
depths as the allocating entry point (sg_run_bfs); depths are integers, so
the comparison is exact.  The file is collected last on purpose."""
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


@pytest.mark.parametrize("directed", [False, True])
def test_noalloc_matches_allocating_bfs_twice(sg, rmat, directed):
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
