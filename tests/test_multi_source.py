"""Batched multi-source BFS: each of the k depth rows equals the single-source
BFS from that source (bit-exact), for push, pull and hybrid schedules."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,perm", [(10, 0), (14, 6), (16, 0)])
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_msbfs_matches_oracle(sg, oracle, rmat, scale, perm, direction):
    g = rmat(scale, perm_seed=perm)
    G = sg.graph.build.fromCSR(g)
    srcs = sg.io.sample_sources(g, 64, seed=3)
    mb = sg.algorithms.MultiBFS(G)
    det = mb.run(srcs, direction, 15.0, 24.0)
    d = mb.getDistances()
    ref = oracle.bfs_multi(g, srcs)
    assert np.array_equal(d, ref)
    want_edges = sum(oracle.visited_edges(g, ref[i], g.n + 1) for i in range(len(srcs)))
    assert det["reached_edges"] == want_edges


@pytest.mark.parametrize("k", [1, 7, 33, 64])
def test_msbfs_batch_sizes_and_duplicates(sg, oracle, rmat, k):
    g = rmat(12, perm_seed=1)
    G = sg.graph.build.fromCSR(g)
    rng = np.random.default_rng(k)
    srcs = rng.integers(0, g.n, k).astype(np.uint32)
    if k > 2:
        srcs[1] = srcs[0]  # a repeated source is two independent traversals
    mb = sg.algorithms.MultiBFS(G, 64)
    mb.run(srcs)
    assert np.array_equal(mb.getDistances(), oracle.bfs_multi(g, srcs))


def test_msbfs_directed_and_star(sg, oracle):
    rng = np.random.default_rng(2)
    n = 4000
    g = sg.io.fromCOO(n, rng.integers(0, n, 20000), rng.integers(0, n, 20000), dedupe=True, drop_self_loops=True)
    G = sg.graph.build.fromCSR(g, sg.Properties(directed=True))
    srcs = rng.integers(0, n, 40).astype(np.uint32)
    for direction in (0, 1, 2):
        mb = sg.algorithms.MultiBFS(G)
        mb.run(srcs, direction, 2.0, 4.0)
        assert np.array_equal(mb.getDistances(), oracle.bfs_multi(g, srcs))
    star = sg.io.fromCOO(200_000, np.zeros(199_999, np.uint32), np.arange(1, 200_000, dtype=np.uint32),
                         symmetrize=True)
    Gs = sg.graph.build.fromCSR(star)
    s2 = np.array([0, 5, 77, 199_998], np.uint32)
    mb = sg.algorithms.MultiBFS(Gs, 8)
    mb.run(s2)
    assert np.array_equal(mb.getDistances(), oracle.bfs_multi(star, s2))


@pytest.mark.parametrize("n", [3000, 70_000])
def test_msbfs_long_diameter_depth_planes(sg, oracle, n):
    """Depths above 2^12 and 2^16 (wider depth bit-plane sets), and a second
    batch on the same instance after a deeper one left its planes dirty."""
    path = sg.io.fromCOO(n, np.arange(n - 1), np.arange(1, n), symmetrize=True)
    G = sg.graph.build.fromCSR(path)
    mb = sg.algorithms.MultiBFS(G, 64)
    srcs = np.array([0, n - 1, n // 2, 17], np.uint32)
    for direction in (0, 2):
        det = mb.run(srcs, direction, 15.0, 24.0)
        assert np.array_equal(mb.getDistances(), oracle.bfs_multi(path, srcs))
        assert det["iterations"] == n
    shallow = np.array([n // 2, n // 2 + 1], np.uint32)
    mb.run(shallow)
    assert np.array_equal(mb.getDistances(), oracle.bfs_multi(path, shallow))
