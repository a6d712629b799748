"""Operator layer on the GPU: the reference's operator / frontier known-answer
tests (tests/operators/*.cpp, tests/frontier/mlb_frontier.cpp) ported through
the C ABI, plus randomised checks of every direction x load balancer against
a Python restatement of the advance semantics (operators/advance/common.hpp:49-75)."""
import numpy as np
import pytest

from test_oracle_kat import case, csr_of

pytestmark = pytest.mark.gpu

LBS = [0, 1, 2, 3]


@pytest.fixture(scope="module")
def ops(sg):
    return sg.operators


def test_mlb_frontier_kat(sg, golden):
    c = case(golden, "mlb_frontier")
    G = sg.graph.build.fromCSR(csr_of(sg, golden, c["matrix"]))
    f = sg.frontier.makeFrontier(G)
    for v in c["inserts"]:
        f.insert(v)
    assert f.active() == c["after_insert"]
    saved = f.saveState()
    for v in c["removes"]:
        f.remove(v)
    assert f.active() == c["after_remove"]
    f.clear()
    assert f.empty()
    f.loadState(saved)
    assert f.active() == c["after_load"]
    assert f.size() == len(c["after_load"])
    assert f.check(1) and not f.check(0)


@pytest.mark.parametrize("lb", [2, 3])
def test_advance_push_bfs_kat(sg, ops, golden, lb):
    """tests/operators/advance.cpp: BFS by repeated push advances."""
    c = case(golden, "advance_push_bfs_depths")
    G = sg.graph.build.fromCSR(csr_of(sg, golden, c["matrix"]))
    n = G.getVertexCount()
    fin, fout = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
    visited = sg.DeviceArray(np.zeros(n, np.uint8))
    dist = sg.DeviceArray(np.zeros(n, np.uint64))
    fin.insert(0)
    visited.upload(np.eye(1, n, 0, dtype=np.uint8)[0])
    args = ops.op_args([visited, dist])
    while not fin.empty():
        ops.advance.frontier(G, fin, fout, ops.OP_BFS_VISIT_FLAG, args, ops.direction.push, lb)
        sg.frontier.swap(fin, fout)
        fout.clear()
    assert visited.numpy().all()
    assert dist.numpy().tolist() == c["expected"]


@pytest.mark.parametrize("lb", [2, 3])
def test_advance_graph_kat(sg, ops, golden, lb):
    """tests/operators/advance_graph.cpp: advance::vertices marks degree != 0."""
    c = case(golden, "advance_graph_nonzero_degree")
    G = sg.graph.build.fromCSR(csr_of(sg, golden, c["matrix"]))
    out = sg.frontier.makeFrontier(G)
    ops.advance.vertices(G, out, ops.OP_NONZERO_DEGREE, None, lb)
    assert out.flags().tolist() == c["expected"]


def test_advance_pull_kat(sg, ops, golden):
    """tests/operators/advance_pull.cpp: in = {0,1}; pull with
    infer_from_device; both LBs agree; bucketing visits vertex 2 once."""
    c = case(golden, "advance_pull_short_circuit")
    G = sg.graph.build.fromCSR(csr_of(sg, golden, c["matrix"]))
    n = G.getVertexCount()
    result = {}
    for lb in (2, 3):
        fin, fout = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
        for v in c["in_frontier"]:
            fin.insert(v)
        visits = sg.DeviceArray(np.zeros(n, np.uint32))
        ops.advance.frontier(G, fin, fout, ops.OP_COUNT_VISITS, ops.op_args([visits]), ops.direction.pull, lb,
                             expected_size=ops.size.infer_from_device)
        active = sg.DeviceArray(np.zeros(n, np.uint8))
        ops.compute.execute(G, fout, ops.FN_SET_U8, ops.op_args([active]))
        result[lb] = (visits.numpy()[2], active.numpy())
    assert np.array_equal(result[2][1], result[3][1])
    assert result[2][1][2] == 1
    assert result[2][0] >= c["workgroup_visits_of_2_at_least"]
    assert result[3][0] == c["bucketing_visits_of_2"]


def test_filter_compute_kat(sg, ops, golden):
    """tests/operators/filter_compute.cpp on star_5."""
    c = case(golden, "filter_compute")
    G = sg.graph.build.fromCSR(csr_of(sg, golden, c["matrix"]))
    inp, out = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
    for v in c["input"]:
        inp.insert(v)
    ops.filter.external(G, inp, out, ops.PRED_EVEN)
    assert out.active() == c["external_even"]
    ops.filter.inplace(G, inp, ops.PRED_LESS_THAN, ops.op_args(u=[c["inplace_remove_less_than"]]))
    assert inp.active() == c["after_inplace"]
    seen = sg.DeviceArray(np.zeros(G.getVertexCount(), np.uint32))
    ops.compute.execute(G, out, ops.FN_MARK, ops.op_args([seen]))
    assert seen.numpy().tolist() == c["execute_seen"]
    assert ops.compute.reduce(G, out, ops.RED_VERTEX_ID) == c["reduce_sum"]


def test_intersection_kat(sg, ops, golden):
    c = case(golden, "intersection")
    G = sg.graph.build.fromCSR(csr_of(sg, golden, c["matrix"]))
    a, b, o = (sg.frontier.makeFrontier(G) for _ in range(3))
    for v in c["lhs"]:
        a.insert(v)
    for v in c["rhs"]:
        b.insert(v)
    ops.intersection.execute(G, a, b, o)
    assert o.active() == c["expected"]


def test_unsupported_load_balancer(sg, ops, golden):
    G = sg.graph.build.fromCSR(csr_of(sg, golden, "line_5"))
    f = sg.frontier.makeFrontier(G)
    with pytest.raises(sg._lib.SygraphError) as ei:
        ops.advance.frontier(G, f, f, ops.OP_TRUE, None, ops.direction.push, 7)
    assert ei.value.status == sg._lib.SG_ERR_UNSUPPORTED


def reference_advance(ro, col, in_flags, direction):
    """Python restatement of one advance with an always-true functor:
    push -> out = neighbours of the frontier; pull / pull_all -> out = the
    vertices outside the frontier with a neighbour inside it."""
    n = in_flags.size
    out = np.zeros(n, np.uint8)
    if direction == 0:
        for v in np.nonzero(in_flags)[0]:
            out[col[ro[v]:ro[v + 1]]] = 1
    else:
        for v in range(n):
            if in_flags[v]:
                continue
            if in_flags[col[ro[v]:ro[v + 1]]].any():
                out[v] = 1
    return out


@pytest.mark.parametrize("lb", LBS)
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_advance_random_frontiers(sg, ops, rmat, lb, direction):
    g = rmat(11, perm_seed=3)
    G = sg.graph.build.fromCSR(g)
    rng = np.random.default_rng(lb * 10 + direction)
    for density in (0.001, 0.05, 0.5):
        flags = (rng.random(g.n) < density).astype(np.uint8)
        fin, fout = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
        fin.insert_list(np.nonzero(flags)[0])
        ops.advance.frontier(G, fin, fout, ops.OP_TRUE, None, direction, lb)
        assert np.array_equal(fout.flags(), reference_advance(g.row_offsets, g.column_indices, flags, direction))


@pytest.mark.parametrize("lb", LBS)
def test_advance_pull_visit_counts(sg, ops, rmat, lb):
    """pull short-circuits after the first success (each activated candidate
    visited at least once, bucketing's lane bucket exactly once); pull_all
    visits every in-frontier neighbour."""
    g = rmat(10, perm_seed=5)
    G = sg.graph.build.fromCSR(g)
    rng = np.random.default_rng(lb)
    flags = (rng.random(g.n) < 0.1).astype(np.uint8)
    ro, col = g.row_offsets, g.column_indices
    expect_all = np.array([0 if flags[v] else int(flags[col[ro[v]:ro[v + 1]]].sum()) for v in range(g.n)])
    for direction in (1, 2):
        fin, fout = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
        fin.insert_list(np.nonzero(flags)[0])
        visits = sg.DeviceArray(np.zeros(g.n, np.uint32))
        ops.advance.frontier(G, fin, fout, ops.OP_COUNT_VISITS, ops.op_args([visits]), direction, lb)
        got = visits.numpy()
        if direction == 2:
            assert np.array_equal(got, expect_all)
        else:
            assert np.array_equal(got > 0, expect_all > 0)
            assert (got <= expect_all).all()
            if lb == 0:
                assert np.array_equal(got, np.minimum(expect_all, 1))


def test_advance_bfs_ops_match_engine(sg, ops, oracle, rmat):
    """A BFS written with the reference's push / pull functors through
    sg_advance gives the oracle's depths (the plain operator-level loop)."""
    g = rmat(12, perm_seed=9)
    G = sg.graph.build.fromCSR(g)
    n = g.n
    src = int(np.argmax(g.degrees()))
    for direction in (0, 1):
        depth = sg.DeviceArray(np.full(n, n + 1, np.uint32))
        d0 = np.full(n, n + 1, np.uint32)
        d0[src] = 0
        depth.upload(d0)
        fin, fout = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
        fin.insert(src)
        it = 0
        while not fin.empty():
            op = ops.OP_BFS_PUSH if direction == 0 else ops.OP_BFS_PULL
            ops.advance.frontier(G, fin, fout, op, ops.op_args([depth], [n + 1, it]), direction, 2)
            sg.frontier.swap(fin, fout)
            fout.clear()
            it += 1
        assert np.array_equal(depth.numpy(), oracle.bfs_levels(g, src))


def test_sssp_relax_op_reaches_dijkstra(sg, ops, oracle, rmat):
    g = rmat(10, perm_seed=2)
    G = sg.graph.build.fromCSR(g)
    n, src = g.n, 5
    d0 = np.full(n, n + 1, np.float32)
    d0[src] = 0
    dist = sg.DeviceArray(d0)
    fin, fout = sg.frontier.makeFrontier(G), sg.frontier.makeFrontier(G)
    fin.insert(src)
    visited = sg.DeviceArray(np.full(n, -1, np.int32))
    it = 0
    while not fin.empty():
        ops.advance.frontier(G, fin, fout, ops.OP_SSSP_RELAX, ops.op_args([dist]), 0, 2)
        ops.filter.external(G, fout, fin, ops.PRED_ITER_MARK, ops.op_args([visited], [it]))
        fout.clear()
        it += 1
    assert np.array_equal(dist.numpy(), oracle.sssp_dijkstra(g, src))


def test_compute_reduce_degree_and_segmented_intersection(sg, ops, rmat, oracle):
    g = rmat(10, perm_seed=4)
    G = sg.graph.build.fromCSR(g)
    f = sg.frontier.makeFrontier(G)
    ids = np.arange(0, g.n, 7)
    f.insert_list(ids)
    assert ops.compute.reduce(G, f, ops.RED_DEGREE) == int(g.degrees()[ids].sum())
    assert ops.compute.reduce(G, f, ops.RED_COUNT) == ids.size
    rng = np.random.default_rng(1)
    a = rng.integers(0, g.n, 500).astype(np.uint32)
    b = rng.integers(0, g.n, 500).astype(np.uint32)
    got = ops.segmented_intersection(G, a, b)
    ro, col = g.row_offsets, g.column_indices
    want = [len(np.intersect1d(col[ro[x]:ro[x + 1]], col[ro[y]:ro[y + 1]])) for x, y in zip(a, b)]
    assert got.tolist() == want
