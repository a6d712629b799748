"""Batched BC (64 sources per launch, bit-parallel frontiers) against the
FP64 Brandes oracle within 1e-4 relative, bit-identical across repeated
runs, and through the history-enlarging path for deep graphs."""
import numpy as np
import pytest

from test_oracle_kat import case, csr_of

pytestmark = pytest.mark.gpu

BC_RTOL = 1e-4


def _check(got, ref):
    got = got.astype(np.float64)
    np.testing.assert_allclose(got, ref, rtol=BC_RTOL, atol=BC_RTOL * max(1.0, float(np.abs(ref).max())) * 1e-3)


def test_batched_bc_line5(sg, golden):
    G = sg.graph.build.fromCSR(csr_of(sg, golden, "line_5"))
    bc = sg.algorithms.BatchedBC(G)
    bc.run([case(golden, "bc_line5_runs")["source"]])
    np.testing.assert_allclose(bc.getBC(), [0, 3, 2, 1, 0], rtol=BC_RTOL)


@pytest.mark.parametrize("scale,perm,k", [(10, 0, 64), (13, 5, 64), (16, 0, 100), (12, 3, 1)])
def test_batched_bc_rmat(sg, oracle, rmat, scale, perm, k):
    g = rmat(scale, perm_seed=perm)
    srcs = sg.io.sample_sources(g, k, seed=3)
    bc = sg.algorithms.BatchedBC(sg.graph.build.fromCSR(g))
    det = bc.run(srcs)
    _check(bc.getBC(), oracle.bc(g, srcs))
    want = sum(oracle.visited_edges(g, oracle.bfs_levels(g, int(s)), g.n + 1) for s in srcs)
    assert det["reached_edges"] == want


def test_batched_bc_is_deterministic_and_matches_per_source(sg, oracle, rmat):
    g = rmat(14, perm_seed=1)
    G = sg.graph.build.fromCSR(g)
    srcs = sg.io.sample_sources(g, 64, seed=9)
    a = sg.algorithms.BatchedBC(G)
    a.run(srcs)
    x = a.getBC()
    a.run(srcs)
    assert np.array_equal(x.view(np.uint32), a.getBC().view(np.uint32))
    b = sg.algorithms.BC(G)
    b.init(srcs)
    b.run()
    _check(x, b.getBC().astype(np.float64))
    # sg_bc_batched (one-shot) gives the same bits as the instance API
    import ctypes as C
    out = np.empty(g.n, np.float32)
    s32 = np.ascontiguousarray(srcs, np.uint32)
    sg._lib.call("sg_bc_batched", G.handle, s32.ctypes.data_as(C.POINTER(C.c_uint32)), s32.size,
                 out.ctypes.data_as(C.POINTER(C.c_float)))
    assert np.array_equal(out.view(np.uint32), x.view(np.uint32))


def test_batched_bc_directed_duplicates_and_hubs(sg, oracle):
    rng = np.random.default_rng(4)
    n = 5000
    # a few hubs with in/out-degree above the CTA threshold plus random arcs
    hubs = rng.integers(0, n, 4)
    src = np.concatenate([rng.integers(0, n, 30000), np.repeat(hubs, 3000), rng.integers(0, n, 12000)])
    dst = np.concatenate([rng.integers(0, n, 30000), rng.integers(0, n, 12000), np.repeat(hubs, 3000)])
    g = sg.io.fromCOO(n, src, dst, dedupe=True, drop_self_loops=True)
    G = sg.graph.build.fromCSR(g, sg.Properties(directed=True))
    srcs = np.concatenate([hubs, rng.integers(0, n, 40)]).astype(np.uint32)
    srcs[5] = srcs[4]  # a repeated source counts twice
    bc = sg.algorithms.BatchedBC(G)
    bc.run(srcs)
    _check(bc.getBC(), oracle.bc(g, srcs))


def test_batched_bc_history_grows_for_deep_graphs(sg, oracle):
    n = 3000
    path = sg.io.fromCOO(n, np.arange(n - 1), np.arange(1, n), symmetrize=True)
    G = sg.graph.build.fromCSR(path)
    bc = sg.algorithms.BatchedBC(G, history_levels=4)
    srcs = np.array([0, n // 3, n - 1], np.uint32)
    det = bc.run(srcs)
    assert det["history_retries"] >= 1 and det["history_levels"] >= n
    _check(bc.getBC(), oracle.bc(path, srcs))
    # accumulate: a second batch adds to the first
    bc.run(srcs[:1], accumulate=True)
    _check(bc.getBC(), oracle.bc(path, np.concatenate([srcs, srcs[:1]])))
