"""Oracle parity on the benchmark inputs themselves, not only on small graphs.

The reference validates every example run on its benchmark graph against a
CPU BFS and a CPU Dijkstra (examples/bfs/bfs.cpp:16-56,
examples/sssp/sssp.cpp:23-66).  These tests do the same on the graphs and
sources the benchmarks time:

* RMAT-22 (seed 1, float32 weights seed 2) and the bench's 64 sources (seed 3):
  hybrid BFS (alpha 15, beta 24) against oracle.bfs_frontier -- depths,
  iterations and the push / pull step sets; SSSP by the reference's frontier
  Bellman-Ford and by delta-stepping against oracle.sssp_dijkstra, fp32 bits;
  the 64 sources as one batched launch against oracle.bfs_multi.
* RMAT-20: batched Brandes BC (64 sources) within 1e-4 relative of the FP64
  oracle; CC (union-find and propagation) against the max-label fixed point;
  TC against the DAG count.
* The selector's evaluation graphs, RMAT-23 and the 4096 x 4096 grid with 2%
  long-range pairs (uint32 weights on [1,64]): learned-mode BFS against the
  oracle, and SSSP against Dijkstra.

Integers and distances are compared bit for bit; BC within BC_RTOL."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

BC_RTOL = 1e-4
ALPHA, BETA = 15.0, 24.0


@pytest.fixture(scope="module")
def rmat22(sg):
    g = sg.io.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, weight_seed=2, perm_seed=0, value_type=sg.WEIGHT_F32)
    return g, sg.graph.build.fromCSR(g), sg.io.sample_sources(g, 64, seed=3)


@pytest.fixture(scope="module")
def rmat20(sg):
    g = sg.io.rmat(20, 16, 0.57, 0.19, 0.19, seed=1)
    return g, sg.graph.build.fromCSR(g), sg.io.sample_sources(g, 64, seed=3)


def test_bfs_rmat22_bench_sources(sg, oracle, rmat22):
    g, G, srcs = rmat22
    bfs = sg.algorithms.BFS(G)
    for s in srcs[:4]:
        bfs.init(int(s))
        det = bfs.run(sg.algorithms.bfs_direction.hybrid, ALPHA, BETA)
        want, it, steps = oracle.bfs_frontier(g, int(s), 2, ALPHA, BETA)
        assert np.array_equal(bfs.getDistances(), want), int(s)
        assert det.iterations == it
        assert det.pull_steps == {i for i, p in enumerate(steps) if p}
        assert det.push_steps == {i for i, p in enumerate(steps) if not p}
        assert det.visited_edges == oracle.visited_edges(g, want, g.n + 1)


@pytest.mark.parametrize("delta", [0.0, 0.1])
def test_sssp_rmat22_bench_sources(sg, oracle, rmat22, delta):
    g, G, srcs = rmat22
    sssp = sg.algorithms.SSSP(G)
    sssp.set_delta(delta)
    for s in srcs[:4]:
        sssp.init(int(s))
        sssp.run()
        want = oracle.sssp_dijkstra(g, int(s))
        assert np.array_equal(sssp.getDistances().view(np.uint32), want.view(np.uint32)), (delta, int(s))


def test_multibfs_rmat22_all_bench_sources(sg, oracle, rmat22):
    g, G, srcs = rmat22
    mb = sg.algorithms.MultiBFS(G, 64)
    mb.run(srcs, sg.algorithms.bfs_direction.hybrid, 4.0, 24.0)
    got = mb.getDistances()
    want = oracle.bfs_multi(g, srcs)
    for i in range(64):
        assert np.array_equal(got[i], want[i]), i


def test_batched_bc_rmat20(sg, oracle, rmat20):
    g, G, srcs = rmat20
    bc = sg.algorithms.BatchedBC(G)
    bc.run(srcs)
    ref = oracle.bc(g, srcs)
    np.testing.assert_allclose(bc.getBC(), ref, rtol=BC_RTOL, atol=BC_RTOL * max(1.0, float(ref.max())) * 1e-3)


def test_cc_rmat20(sg, oracle, rmat20):
    g, G, _ = rmat20
    want = oracle.cc_maxlabel(g)
    cc = sg.algorithms.CC(G)
    for method in (cc.AUTO, cc.PROPAGATION):
        cc.set_method(method)
        cc.run()
        assert np.array_equal(cc.getLabels(), want), method


def test_tc_rmat20(sg, oracle, rmat20):
    g, G, _ = rmat20
    tc = sg.algorithms.TC(G)
    tc.run()
    total, _ = oracle.tc_dag(g)
    assert tc.getNumTriangles() == total


def _selector_graphs(sg):
    yield "rmat23", sg.io.rmat(23, 16, 0.57, 0.19, 0.19, seed=1, weight_seed=2, value_type=sg.WEIGHT_U32)
    yield "grid4096", sg.io.grid(4096, long_range_frac=0.02, seed=103, weight_seed=2, value_type=sg.WEIGHT_U32)


def test_learned_selector_graphs(sg, oracle):
    """The three learned modes on the selector's evaluation graphs against the
    oracle: single-source BFS, delta-stepping SSSP with the learned heavy
    phases, and the batched BFS (8 sources) with its model."""
    from sygraph_b200 import selector, train_selector
    mlp = selector.Mlp.load()
    sssp_mlp = selector.Mlp.load(train_selector.SSSP_MODEL_PATH)
    batch_mlp = selector.Mlp.load(train_selector.BATCHED_MODEL_PATH)
    for name, g in _selector_graphs(sg):
        G = sg.graph.build.fromCSR(g)
        bfs = sg.algorithms.BFS(G)
        bfs.set_selector(mlp)
        sssp = sg.algorithms.SSSP(G)
        sssp.set_selector(sssp_mlp)
        mb = sg.algorithms.MultiBFS(G, 8)
        mb.set_selector(batch_mlp)
        ms = sg.io.sample_sources(g, 8, seed=5)
        mb.run(ms, sg.algorithms.bfs_direction.learned, train_selector.BATCH_ALPHA, train_selector.BATCH_BETA)
        assert np.array_equal(mb.getDistances(), oracle.bfs_multi(g, ms)), name
        del mb
        srcs = sg.io.sample_sources(g, 2, seed=3)
        for s in srcs:
            want, it, _ = oracle.bfs_frontier(g, int(s), 2, ALPHA, BETA)
            bfs.init(int(s))
            det = bfs.run(sg.algorithms.bfs_direction.learned, ALPHA, BETA)
            assert np.array_equal(bfs.getDistances(), want), (name, int(s))
            assert det.iterations == it
            dref = oracle.sssp_dijkstra(g, int(s))
            for delta in (0, 64 if name == "rmat23" else 512):
                sssp.set_delta(delta)
                sssp.init(int(s))
                sssp.run()
                assert np.array_equal(sssp.getDistances(), dref), (name, int(s), delta)
        del bfs, sssp, G
