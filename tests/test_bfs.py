"""BFS parity: the fused CUDA engine against the oracle, bit-exact depths and
the reference's BFSRunDetails (iterations, push / pull step sets)."""
import numpy as np
import pytest

from test_oracle_kat import case, csr_of

pytestmark = pytest.mark.gpu


def run_bfs(sg, csr, source, direction, alpha=1.0, beta=1.0, properties=None):
    G = sg.graph.build.fromCSR(csr, properties)
    bfs = sg.algorithms.BFS(G)
    bfs.init(source)
    det = bfs.run(direction, alpha, beta)
    return bfs.getDistances(), det


def test_bfs_kat_line5(sg, golden):
    c = case(golden, "bfs_line5")
    g = csr_of(sg, golden, c["matrix"])
    D = sg.algorithms.bfs_direction
    d, det = run_bfs(sg, g, 0, D.push)
    assert d.tolist() == c["expected_push"] and det.push_steps and not det.pull_steps
    d, det = run_bfs(sg, g, 0, D.pull)
    assert d.tolist() == c["expected_pull"] and det.pull_steps and not det.push_steps
    d, det = run_bfs(sg, g, 0, D.hybrid, c["hybrid_alpha"], c["hybrid_beta"])
    assert d.tolist() == c["expected_hybrid"]
    assert det.iterations == c["hybrid_iterations"]


def test_bfs_kat_symmetric6(sg, golden):
    c = case(golden, "advance_push_bfs_depths")
    g = csr_of(sg, golden, c["matrix"])
    for direction in (0, 1, 2):
        d, _ = run_bfs(sg, g, c["source"], direction)
        assert d.tolist() == c["expected"]


def test_bfs_init_before_run_and_errors(sg, golden):
    g = csr_of(sg, golden, "line_5")
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    with pytest.raises(sg._lib.SygraphError) as ei:
        bfs.run()
    assert ei.value.status == sg._lib.SG_ERR_NOT_INITIALIZED
    bfs.init(2)
    assert bfs.getDistances().tolist() == [6, 6, 0, 6, 6]
    with pytest.raises(sg._lib.SygraphError):
        bfs.init(5)


@pytest.mark.parametrize("scale,perm", [(10, 0), (14, 7), (16, 0)])
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_bfs_rmat_parity(sg, oracle, rmat, scale, perm, direction):
    g = rmat(scale, perm_seed=perm)
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    srcs = [int(np.argmax(g.degrees()))] + [int(s) for s in sg.io.sample_sources(g, 3, seed=3)]
    for s in srcs:
        bfs.init(s)
        det = bfs.run(direction, 15.0, 24.0)
        d = bfs.getDistances()
        ref, it, steps = oracle.bfs_frontier(g, s, direction, 15.0, 24.0)
        assert np.array_equal(d, ref), f"depth mismatch from source {s}"
        assert det.iterations == it
        assert sorted(det.pull_steps) == [i for i, x in enumerate(steps) if x == 1]
        assert sorted(det.push_steps) == [i for i, x in enumerate(steps) if x == 0]
        assert det.visited_edges == oracle.visited_edges(g, ref, g.n + 1)
        assert det.visited_vertices == int((ref != g.n + 1).sum())


def test_bfs_directed_graph_uses_inverse(sg, oracle):
    rng = np.random.default_rng(5)
    n = 3000
    src = rng.integers(0, n, 20000)
    dst = rng.integers(0, n, 20000)
    g = sg.io.fromCOO(n, src, dst, dedupe=True, drop_self_loops=True)
    props = sg.Properties(directed=True)
    inv = g.invert()
    s0 = int(np.argmax(g.degrees()))
    for direction in (0, 1, 2):
        d, det = run_bfs(sg, g, s0, direction, 2.0, 4.0, props)
        ref, it, _ = oracle.bfs_frontier(g, s0, direction, 2.0, 4.0, inverse=inv)
        assert np.array_equal(d, ref)
        assert det.iterations == it


def test_bfs_edge_cases(sg, oracle):
    # isolated source, single vertex graph, long path (many levels)
    g = sg.io.fromCOO(4, [0, 1], [1, 0])
    d, det = run_bfs(sg, g, 3, 2)
    assert d.tolist() == [5, 5, 5, 0] and det.iterations == 1
    g1 = sg.CSR(np.array([0, 0], np.uint32), np.zeros(0, np.uint32))
    d, det = run_bfs(sg, g1, 0, 0)
    assert d.tolist() == [0]
    n = 5000
    path = sg.io.fromCOO(n, np.arange(n - 1), np.arange(1, n), symmetrize=True)
    for direction in (0, 1, 2):
        d, det = run_bfs(sg, path, 0, direction, 15.0, 24.0)
        assert d.tolist() == list(range(n))
        assert det.iterations == n


def test_bfs_star_hub(sg, oracle):
    """One vertex with a huge degree exercises the chunked expansion."""
    n = 300_000
    src = np.zeros(n - 1, np.uint32)
    dst = np.arange(1, n, dtype=np.uint32)
    g = sg.io.fromCOO(n, src, dst, symmetrize=True)
    for s in (0, 17):
        for direction in (0, 1, 2):
            d, _ = run_bfs(sg, g, s, direction, 15.0, 24.0)
            assert np.array_equal(d, oracle.bfs_levels(g, s))


@pytest.mark.parametrize("directed", [False, True])
def test_bfs_consecutive_runs_across_components(sg, oracle, directed):
    """One instance, sources in components of different sizes and on an
    isolated vertex, in turn, with distances read before a run in between:
    every run gives the oracle's depths (the engine rewrites only the depths
    that the previous run reached and this one does not)."""
    rng = np.random.default_rng(11)
    n = 40_000
    # a big random component on [0, 30000), a path on [30000, 30500), a star
    # on [31000, 31200), the rest isolated
    a = rng.integers(0, 30_000, 150_000)
    b = rng.integers(0, 30_000, 150_000)
    p = np.arange(30_000, 30_499)
    s = np.full(199, 31_000)
    src = np.concatenate([a, p, s])
    dst = np.concatenate([b, p + 1, np.arange(31_001, 31_200)])
    g = sg.io.fromCOO(n, src, dst, symmetrize=not directed, dedupe=True, drop_self_loops=True)
    G = sg.graph.build.fromCSR(g, sg.Properties(directed=True)) if directed else sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    order = [5, 30_000, 123, 31_000, 39_999, 30_250, 7, 31_100, 77, 39_000]
    for k, s0 in enumerate(order):
        bfs.init(s0)
        if k == 4:
            bfs.getDistances()  # the initial state, written before the run
        bfs.run(sg.algorithms.bfs_direction.hybrid, 15.0, 24.0)
        assert np.array_equal(bfs.getDistances(), oracle.bfs_levels(g, s0)), (directed, s0)
