"""SSSP / CC / BC / TC parity on the GPU against the oracle.

SSSP distances, CC labels and TC counts are bit-exact; BC (float32 on the
GPU) is within 1e-4 relative of the FP64 Brandes oracle."""
import numpy as np
import pytest

from test_oracle_kat import case, csr_of

pytestmark = pytest.mark.gpu

BC_RTOL = 1e-4


def test_sssp_kat(sg, golden):
    c = case(golden, "sssp_weighted_directed5")
    for vt in (sg.WEIGHT_U32, sg.WEIGHT_F32):
        g = csr_of(sg, golden, c["matrix"], directed=True, value_type=vt)
        G = sg.graph.build.fromCSR(g)
        s = sg.algorithms.SSSP(G)
        s.init(c["source"])
        s.run()
        assert s.getDistances().tolist() == c["expected"]


@pytest.mark.parametrize("scale,perm", [(10, 0), (14, 3), (16, 0)])
def test_sssp_rmat_f32(sg, oracle, rmat, scale, perm):
    g = rmat(scale, perm_seed=perm)
    G = sg.graph.build.fromCSR(g)
    s = sg.algorithms.SSSP(G)
    for src in [int(np.argmax(g.degrees()))] + [int(x) for x in sg.io.sample_sources(g, 2, seed=4)]:
        s.init(src)
        s.run()
        d = s.getDistances()
        ref = oracle.sssp_dijkstra(g, src)
        assert np.array_equal(d.view(np.uint32), ref.view(np.uint32)), f"distance bits differ from source {src}"


def test_sssp_u32_grid(sg, oracle):
    g = sg.io.grid(64, 0.02, seed=1, weight_seed=2, value_type=sg.WEIGHT_U32)
    G = sg.graph.build.fromCSR(g)
    s = sg.algorithms.SSSP(G)
    for src in (0, 2080):
        s.init(src)
        s.run()
        assert np.array_equal(s.getDistances(), oracle.sssp_dijkstra(g, src))


def test_sssp_unreachable_and_directed(sg, oracle):
    rng = np.random.default_rng(3)
    n = 2000
    src = rng.integers(0, n, 6000)
    dst = rng.integers(0, n, 6000)
    w = (rng.integers(1, 1 << 24, 6000) / float(1 << 24)).astype(np.float32)
    g = sg.io.fromCOO(n, src, dst, w, dedupe=True, drop_self_loops=True)
    G = sg.graph.build.fromCSR(g, sg.Properties(directed=True, weighted=True))
    s = sg.algorithms.SSSP(G)
    s.init(7)
    s.run()
    ref = oracle.sssp_dijkstra(g, 7)
    assert np.array_equal(s.getDistances(), ref)
    assert (ref == np.float32(n + 1)).any()


def test_cc_two_cc(sg, golden):
    G = sg.graph.build.fromCSR(csr_of(sg, golden, "two_cc"))
    cc = sg.algorithms.CC(G)
    for source in case(golden, "cc_two_cc_runs")["sources"]:
        cc.init(source)
        cc.run()
        assert cc.getLabels().tolist() == [4, 4, 4, 4, 4, 5]


@pytest.mark.parametrize("scale,perm", [(10, 0), (14, 11), (16, 0)])
def test_cc_rmat(sg, oracle, rmat, scale, perm):
    g = rmat(scale, perm_seed=perm)
    cc = sg.algorithms.CC(sg.graph.build.fromCSR(g))
    cc.run()
    assert np.array_equal(cc.getLabels(), oracle.cc_maxlabel(g))


def test_cc_directed_reachability(sg, oracle):
    rng = np.random.default_rng(9)
    n = 3000
    g = sg.io.fromCOO(n, rng.integers(0, n, 5000), rng.integers(0, n, 5000), dedupe=True, drop_self_loops=True)
    cc = sg.algorithms.CC(sg.graph.build.fromCSR(g, sg.Properties(directed=True)))
    cc.run()
    assert np.array_equal(cc.getLabels(), oracle.cc_maxlabel(g))


def test_bc_line5(sg, golden):
    G = sg.graph.build.fromCSR(csr_of(sg, golden, "line_5"))
    bc = sg.algorithms.BC(G)
    bc.init(case(golden, "bc_line5_runs")["source"])
    bc.run()
    np.testing.assert_allclose(bc.getBC(), [0, 3, 2, 1, 0], rtol=BC_RTOL)


@pytest.mark.parametrize("scale,perm", [(10, 0), (13, 5)])
def test_bc_rmat(sg, oracle, rmat, scale, perm):
    g = rmat(scale, perm_seed=perm)
    srcs = sg.io.sample_sources(g, 8, seed=3)
    bc = sg.algorithms.BC(sg.graph.build.fromCSR(g))
    bc.init(srcs)
    bc.run()
    ref = oracle.bc(g, srcs)
    got = bc.getBC().astype(np.float64)
    np.testing.assert_allclose(got, ref, rtol=BC_RTOL, atol=BC_RTOL * max(1.0, float(ref.max())) * 1e-3)


def test_tc_kat(sg, golden):
    G = sg.graph.build.fromCSR(csr_of(sg, golden, "triangle_3"))
    tc = sg.algorithms.TC(G)
    tc.init()
    tc.run(per_vertex=True)
    assert tc.getNumTriangles() == case(golden, "tc_triangle3")["expected"]
    assert [tc.getNumTriangles(v) for v in range(3)] == [2, 1, 0]


@pytest.mark.parametrize("scale,perm", [(10, 0), (14, 2), (16, 0)])
def test_tc_rmat(sg, oracle, rmat, scale, perm):
    g = rmat(scale, perm_seed=perm)
    tc = sg.algorithms.TC(sg.graph.build.fromCSR(g))
    tc.run(per_vertex=True)
    tot, pv = oracle.tc_dag(g, per_vertex=True)
    assert tc.getNumTriangles() == tot
    assert np.array_equal(tc.per_vertex, pv)
    if scale <= 10:
        assert oracle.tc_edge_merge(g)[0] == tot
