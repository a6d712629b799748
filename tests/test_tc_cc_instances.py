"""Triangle counting and connected components through their instances, against
the oracle: block-table vertices (DAG out-degree above 128), unsorted rows,
self-loops, graphs without edges, and repeated runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _edges(g):
    ro = g.row_offsets.astype(np.int64)
    return np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(ro)), g.column_indices


def _check_tc(sg, oracle, g):
    tc = sg.algorithms.TC(sg.graph.build.fromCSR(g))
    tc.run(per_vertex=True)
    tot, pv = oracle.tc_dag(g, per_vertex=True)
    assert tc.getNumTriangles() == tot
    assert np.array_equal(tc.per_vertex, pv)
    return tc


def test_tc_clique_block_tables(sg, oracle):
    # K_600: DAG out-degrees 0..599, so block tables and both warp lists count
    k = 600
    iu, ju = np.triu_indices(k, 1)
    g = sg.io.fromCOO(k, iu, ju, symmetrize=True, dedupe=True)
    tc = _check_tc(sg, oracle, g)
    assert tc.getNumTriangles() == k * (k - 1) * (k - 2) // 6


def test_tc_clique_pieces(sg, oracle):
    # K_1100: DAG out-degrees up to 1099 > 1024, so the largest vertices are
    # counted in two pieces of their table, every row streamed against each
    k = 1100
    iu, ju = np.triu_indices(k, 1)
    g = sg.io.fromCOO(k, iu, ju, symmetrize=True, dedupe=True)
    for shorter in (True, False):
        tc = sg.algorithms.TC(sg.graph.build.fromCSR(g))
        tc.set_shorter_rows(shorter)
        tc.run(per_vertex=True)
        assert tc.getNumTriangles() == k * (k - 1) * (k - 2) // 6
        # every vertex of a clique lies in C(k-1, 2) triangles; the per-vertex
        # convention (2 to the lowest id, 1 to the middle one) gives
        # 2*C(k-1-v, 2) + v*(k-1-v) for vertex v
        v = np.arange(k, dtype=np.int64)
        want = 2 * ((k - 1 - v) * (k - 2 - v) // 2) + v * (k - 1 - v)
        assert np.array_equal(tc.per_vertex.astype(np.int64), want)


def test_tc_planted_clique_rmat(sg, oracle, rmat):
    g = rmat(13)
    s, d = _edges(g)
    members = np.random.default_rng(5).choice(g.n, 400, replace=False).astype(np.uint32)
    iu, ju = np.triu_indices(members.size, 1)
    h = sg.io.fromCOO(g.n, np.concatenate([s, members[iu]]), np.concatenate([d, members[ju]]), symmetrize=True,
                      dedupe=True, drop_self_loops=True)
    _check_tc(sg, oracle, h)
    assert oracle.tc_edge_merge(h)[0] == oracle.tc_dag(h)[0]


def test_tc_unsorted_rows(sg, oracle, rmat):
    g = rmat(12)
    ro = g.row_offsets.astype(np.int64)
    col = g.column_indices.copy()
    rng = np.random.default_rng(9)
    for u in range(g.n):
        rng.shuffle(col[ro[u]:ro[u + 1]])
    h = sg.CSR(g.row_offsets, col)
    tc = sg.algorithms.TC(sg.graph.build.fromCSR(h))
    tc.run(per_vertex=True)
    tot, pv = oracle.tc_dag(g, per_vertex=True)
    assert tc.getNumTriangles() == tot
    assert np.array_equal(tc.per_vertex, pv)


def test_tc_self_loops(sg, oracle):
    # self-loops are no DAG edges; parallel edges are outside the definition
    # (the reference's sorted-list merge assumes none either)
    rng = np.random.default_rng(11)
    n = 300
    s = rng.integers(0, n, 6000)
    d = rng.integers(0, n, 6000)
    s[:50] = d[:50]
    g = sg.io.fromCOO(n, s, d, symmetrize=True, dedupe=True)
    assert (g.column_indices == np.repeat(np.arange(n), np.diff(g.row_offsets.astype(np.int64)))).any()
    _check_tc(sg, oracle, g)


@pytest.mark.parametrize("n", [1, 7])
def test_tc_no_edges(sg, n):
    g = sg.CSR(np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32))
    tc = sg.algorithms.TC(sg.graph.build.fromCSR(g))
    tc.run(per_vertex=True)
    assert tc.getNumTriangles() == 0
    assert not tc.per_vertex.any()


def test_tc_instance_reruns(sg, oracle, rmat):
    g = rmat(14, perm_seed=6)
    tot, pv = oracle.tc_dag(g, per_vertex=True)
    tc = sg.algorithms.TC(sg.graph.build.fromCSR(g))
    for per_vertex in (False, True, False, True):
        tc.run(per_vertex=per_vertex)
        assert tc.getNumTriangles() == tot
        if per_vertex:
            assert np.array_equal(tc.per_vertex, pv)
    tc.run_async()
    assert tc.getNumTriangles() == tot


def test_cc_instance_reruns(sg, oracle, rmat):
    g = rmat(14, perm_seed=8)
    ref = oracle.cc_maxlabel(g)
    cc = sg.algorithms.CC(sg.graph.build.fromCSR(g))
    for _ in range(3):
        cc.run()
        assert cc.iterations > 0
        assert np.array_equal(cc.getLabels(), ref)
    cc.run_async()
    assert np.array_equal(cc.labels, ref)


@pytest.mark.parametrize("shorter", [False, True])
def test_tc_row_choice(sg, oracle, rmat, shorter):
    g = rmat(15, perm_seed=4)
    tot, pv = oracle.tc_dag(g, per_vertex=True)
    tc = sg.algorithms.TC(sg.graph.build.fromCSR(g))
    tc.set_shorter_rows(shorter)
    tc.run(per_vertex=True)
    assert tc.getNumTriangles() == tot
    assert np.array_equal(tc.per_vertex, pv)


@pytest.mark.parametrize("method", [0, 1, 2])
def test_cc_methods(sg, oracle, rmat, method):
    for g in (rmat(13, perm_seed=2), sg.io.grid(64, 0.0, seed=1)):
        cc = sg.algorithms.CC(sg.graph.build.fromCSR(g))
        cc.set_method(method)
        cc.run()
        assert np.array_equal(cc.getLabels(), oracle.cc_maxlabel(g))
        if method != 1:
            assert cc.iterations == 1


def test_cc_union_find_many_components(sg, oracle):
    # a forest of paths and isolated vertices: many roots, long chains
    rng = np.random.default_rng(13)
    n = 50000
    perm = rng.permutation(n).astype(np.uint32)
    cut = np.sort(rng.choice(n - 1, 3000, replace=False))
    s, d = perm[:-1], perm[1:]
    keep = np.ones(n - 1, bool)
    keep[cut] = False
    g = sg.io.fromCOO(n, s[keep], d[keep], symmetrize=True, dedupe=True)
    ref = oracle.cc_maxlabel(g)
    cc = sg.algorithms.CC(sg.graph.build.fromCSR(g))
    for _ in range(5):  # the links race; every run must give the same labels
        cc.run()
        assert np.array_equal(cc.getLabels(), ref)


def test_cc_union_find_needs_undirected(sg, rmat):
    cc = sg.algorithms.CC(sg.graph.build.fromCSR(rmat(10), sg.Properties(directed=True)))
    with pytest.raises(Exception):
        cc.set_method(2)
    cc.set_method(0)
    cc.run()
    assert cc.iterations > 1


@pytest.mark.parametrize("shape", ["sorted_path", "reversed_path", "star", "two_hubs"])
def test_cc_union_find_adversarial(sg, oracle, shape):
    # shapes that make long parent chains or hot roots under min-linking
    n = 1 << 20 if shape.endswith("path") else 1 << 16
    ids = np.arange(n, dtype=np.uint32)
    if shape == "sorted_path":
        s, d = ids[:-1], ids[1:]
    elif shape == "reversed_path":
        s, d = ids[1:][::-1], ids[:-1][::-1]
    elif shape == "star":
        s, d = np.zeros(n - 1, np.uint32), ids[1:]
    else:  # two hubs, every other vertex on one of them, the hubs unlinked
        s = np.where(ids[2:] % 2 == 0, 0, 1).astype(np.uint32)
        d = ids[2:]
    g = sg.io.fromCOO(n, s, d, symmetrize=True, dedupe=True)
    # closed forms (the oracle's propagation needs one pass per path vertex)
    if shape == "two_hubs":
        ref = np.where(ids % 2 == 0, n - 2, n - 1).astype(np.uint32)
    else:
        ref = np.full(n, n - 1, np.uint32)
    if n <= 1 << 16:
        assert np.array_equal(oracle.cc_maxlabel(g), ref)
    cc = sg.algorithms.CC(sg.graph.build.fromCSR(g))
    for _ in range(2):
        cc.run()
        assert np.array_equal(cc.getLabels(), ref)
