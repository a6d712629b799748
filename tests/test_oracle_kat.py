"""Pin the oracle against the reference's own known answers (tests/golden/kat.json,
extracted from SYgraph's tests by tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest


def csr_of(sg, golden, name, directed=False, value_type=None):
    m = golden["matrices"][name]
    text = f"{m['n']}\n" + "\n".join(" ".join(map(str, r)) for r in m["rows"])
    vt = value_type if value_type is not None else sg.WEIGHT_U32
    return sg.io.fromMatrix(text, vt, sg.Properties(directed=directed, weighted=True))


def case(golden, name):
    return next(c for c in golden["cases"] if c["name"] == name)


def test_golden_file_has_every_case(golden):
    names = {c["name"] for c in golden["cases"]}
    for need in ("advance_push_bfs_depths", "advance_graph_nonzero_degree", "advance_pull_short_circuit",
                 "filter_compute", "intersection", "mlb_frontier", "bfs_line5", "sssp_weighted_directed5",
                 "tc_triangle3"):
        assert need in names
    assert golden["binary_csr"]["magic"] == 0x5359475243535201


def test_bfs_kat_push_pull_hybrid(sg, oracle, golden):
    c = case(golden, "bfs_line5")
    g = csr_of(sg, golden, c["matrix"])
    d, it, steps = oracle.bfs_frontier(g, c["source"], 0)
    assert d.tolist() == c["expected_push"] and set(steps) == {0}
    d, it, steps = oracle.bfs_frontier(g, c["source"], 1)
    assert d.tolist() == c["expected_pull"] and set(steps) == {1}
    d, it, steps = oracle.bfs_frontier(g, c["source"], 2, c["hybrid_alpha"], c["hybrid_beta"])
    assert d.tolist() == c["expected_hybrid"] and it == c["hybrid_iterations"]
    assert oracle.bfs_levels(g, c["source"]).tolist() == c["expected_push"]


def test_advance_bfs_kat(sg, oracle, golden):
    c = case(golden, "advance_push_bfs_depths")
    g = csr_of(sg, golden, c["matrix"])
    assert oracle.bfs_levels(g, c["source"]).tolist() == c["expected"]


def test_sssp_kat(sg, oracle, golden):
    c = case(golden, "sssp_weighted_directed5")
    g = csr_of(sg, golden, c["matrix"], directed=True)
    assert oracle.sssp_dijkstra(g, c["source"]).tolist() == c["expected"]
    gf = csr_of(sg, golden, c["matrix"], directed=True, value_type=sg.WEIGHT_F32)
    d, _ = oracle.sssp_frontier(gf, c["source"])
    assert d.tolist() == [float(x) for x in c["expected"]]


def test_tc_kat(sg, oracle, golden):
    c = case(golden, "tc_triangle3")
    g = csr_of(sg, golden, c["matrix"])
    tot, pv = oracle.tc_edge_merge(g)
    assert tot == c["expected"]
    assert pv.tolist() == [2, 1, 0]
    assert oracle.tc_dag(g)[0] == c["expected"]


def test_cc_two_cc_max_label(sg, oracle, golden):
    g = csr_of(sg, golden, "two_cc")
    # component {0..4} takes its max id 4, the isolated vertex 5 keeps 5
    assert oracle.cc_maxlabel(g).tolist() == [4, 4, 4, 4, 4, 5]


def test_bc_line5_brandes(sg, oracle, golden):
    g = csr_of(sg, golden, "line_5")
    # path 0-1-2-3-4 from source 0: delta(v) = number of vertices beyond v
    assert oracle.bc(g, [0]).tolist() == [0.0, 3.0, 2.0, 1.0, 0.0]


@pytest.mark.parametrize("scale", [8, 10])
def test_oracle_self_consistency(rmat, oracle, scale):
    """Independent restatements agree: frontier BFS (every direction) vs the
    validator, frontier Bellman-Ford vs Dijkstra, TC merge vs DAG."""
    g = rmat(scale)
    src = int(np.argmax(g.degrees()))
    ref = oracle.bfs_levels(g, src)
    for direction in (0, 1, 2):
        d, _, _ = oracle.bfs_frontier(g, src, direction, 15.0, 24.0)
        assert np.array_equal(d, ref)
    d1 = oracle.sssp_dijkstra(g, src)
    d2, _ = oracle.sssp_frontier(g, src)
    assert np.array_equal(d1, d2)
    assert oracle.tc_edge_merge(g)[0] == oracle.tc_dag(g)[0]
    _, pv = oracle.tc_edge_merge(g)
    _, pv2 = oracle.tc_dag(g, per_vertex=True)
    assert np.array_equal(pv, pv2)


def test_bc_matches_networkx_style_definition(rmat, oracle):
    """Brandes dependencies equal a brute-force count of shortest paths."""
    g = rmat(6)
    n = g.n
    ro, col = g.row_offsets, g.column_indices
    srcs = [0, 3, 7]
    dist = np.full((n, n), -1)
    sigma = np.zeros((n, n))
    for s in range(n):
        dist[s, s] = 0
        sigma[s, s] = 1
        q = [s]
        for v in q:
            for e in range(ro[v], ro[v + 1]):
                u = col[e]
                if dist[s, u] < 0:
                    dist[s, u] = dist[s, v] + 1
                    q.append(u)
                if dist[s, u] == dist[s, v] + 1:
                    sigma[s, u] += sigma[s, v]
    expect = np.zeros(n)
    for s in srcs:
        for t in range(n):
            if t == s or dist[s, t] < 0:
                continue
            for v in range(n):
                if v in (s, t) or dist[s, v] < 0 or dist[v, t] < 0:
                    continue
                if dist[s, v] + dist[v, t] == dist[s, t]:
                    expect[v] += sigma[s, v] * sigma[v, t] / sigma[s, t]
    np.testing.assert_allclose(oracle.bc(g, srcs), expect, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("scale,kw", [(10, {}), (12, {"perm_seed": 7}), (14, {"seed": 5, "weight_seed": 9}),
                                      (11, {"value_type": 2}), (9, {"value_type": 0, "a": 0.45, "b": 0.25,
                                                                     "c": 0.15})])
def test_oracle_rmat_equals_the_product_generator(sg, oracle, scale, kw):
    """The CPU baseline arm builds its graph with the oracle's generator, so
    that it loads nothing of the product: the two generators agree bit for bit."""
    o = oracle.rmat(scale, **kw)
    vt = kw.get("value_type", 1)
    p = sg.io.rmat(scale, **{**kw, "value_type": vt})
    assert np.array_equal(o.row_offsets, p.row_offsets)
    assert np.array_equal(o.column_indices, p.column_indices)
    if vt:
        assert np.array_equal(o.values.view(np.uint32), p.values.view(np.uint32))
    else:
        assert o.values is None
    assert np.array_equal(oracle.sample_sources(o, 64, seed=3), sg.io.sample_sources(p, 64, seed=3))
