"""Serving with continuous batching: every result of a mixed, batched,
overlapped run equals the same query run alone (bit for bit), under memory
budgets that force evictions, batch fallbacks and refusals."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs(sg, rmat):
    g1 = rmat(12, perm_seed=1)
    g2 = rmat(14, perm_seed=2)
    g3 = sg.io.grid(96, 0.02, seed=5, weight_seed=6, value_type=sg.WEIGHT_U32)
    return [g1, g2, g3]


def _alone(sg, G, kind, src, delta):
    if kind == "bfs":
        b = sg.algorithms.BFS(G)
        b.init(src)
        b.run(2, 15.0, 24.0)
        return b.getDistances()
    s = sg.algorithms.SSSP(G)
    s.set_delta(delta)
    s.init(src)
    s.run()
    return s.getDistances()


def _run_mixed(sg, graphs, n_queries, seed, **cfg):
    from sygraph_b200 import serving
    Gs = [sg.graph.build.fromCSR(g) for g in graphs]
    srv = serving.Server(**cfg)
    gids = [srv.add_graph(G) for G in Gs]
    rng = np.random.default_rng(seed)
    qs, outs, tickets = [], [], []
    for _ in range(n_queries):
        gi = int(rng.integers(0, len(graphs)))
        kind = "bfs" if rng.random() < 0.7 else "sssp"
        src = int(rng.integers(0, graphs[gi].n))
        dt = np.uint32 if (kind == "bfs" or graphs[gi].value_type != sg.WEIGHT_F32) else np.float32
        out = serving.PinnedBuffer(graphs[gi].n, dt)
        qs.append((gi, kind, src))
        outs.append(out)
        tickets.append(srv.submit(gids[gi], kind, src, out))
    res = [srv.wait(t) for t in tickets]
    stats = srv.stats()
    srv.close()
    return Gs, qs, outs, res, stats


def test_mixed_results_equal_alone(sg, graphs):
    delta = 0.3
    Gs, qs, outs, res, stats = _run_mixed(sg, graphs, 240, 7, slots=4, sssp_delta=delta)
    assert all(r["status"] == 0 for r in res)
    assert stats["completed"] == 240 and stats["batched_queries"] > 0
    assert max(r["batch_size"] for r in res) > 1
    cache = {}
    for (gi, kind, src), out, r in zip(qs, outs, res):
        key = (gi, kind, src)
        if key not in cache:
            cache[key] = _alone(sg, Gs[gi], kind, src, delta)
        want = cache[key]
        assert np.array_equal(out.array.view(np.uint32), want.view(np.uint32)), key
        assert r["end_ns"] >= r["start_ns"] >= r["submit_ns"]
    # launches of different slots were in flight together: a query's launch
    # is (start_ns, end_ns) -- the queries of one batched launch share it --
    # and some two launches overlap in time
    launches = sorted({(r["start_ns"], r["end_ns"]) for r in res})
    assert len(launches) > 1
    overlapping = sum(1 for (s0, e0), (s1, e1) in zip(launches, launches[1:]) if s1 < e0)
    assert overlapping > 0, launches[:8]


def test_tight_budget_evicts_and_still_matches(sg, graphs):
    # room for about one single-traversal workspace of the largest graph:
    # batches can never fit (single traversals instead), workspaces get evicted
    n = max(g.n for g in graphs)
    budget = 512 * 1024 + 40 * n
    Gs, qs, outs, res, stats = _run_mixed(sg, graphs, 60, 11, slots=2, memory_budget=budget, sssp_delta=0.0)
    assert all(r["status"] == 0 for r in res)
    assert stats["evictions"] > 0 and stats["peak_workspace_bytes"] <= budget
    assert stats["batched_queries"] == 0
    for (gi, kind, src), out in zip(qs, outs):
        assert np.array_equal(out.array.view(np.uint32), _alone(sg, Gs[gi], kind, src, 0.0).view(np.uint32))


def test_workspace_that_never_fits_is_refused(sg, graphs):
    from sygraph_b200 import serving
    G = sg.graph.build.fromCSR(graphs[1])
    srv = serving.Server(slots=1, memory_budget=4096)
    gid = srv.add_graph(G)
    r = srv.wait(srv.submit(gid, "bfs", 0, None))
    assert r["status"] == sg._lib.SG_ERR_NOMEM
    with pytest.raises(sg._lib.SygraphError):
        srv.submit(gid, "bfs", graphs[1].n, None)  # source out of range
    with pytest.raises(sg._lib.SygraphError):
        srv.wait(99)  # unknown ticket
    assert srv.stats()["failed"] == 1
    srv.close()


def test_prepare_builds_every_workspace_before_queries(sg, graphs):
    """After prepare, queries of every kind run without building a workspace
    (the workspace bytes do not grow) and match the single-query results; a
    budget too small for them all is reported, without evicting."""
    from sygraph_b200 import serving
    Gs = [sg.graph.build.fromCSR(g) for g in graphs[:2]]
    srv = serving.Server(slots=2, sssp_delta=0.1)
    gids = [srv.add_graph(G) for G in Gs]
    for gi in gids:
        srv.prepare(gi)
        srv.prepare(gi)  # a second call finds them all
    before = srv.stats()["workspace_bytes"]
    assert before > 0
    rng = np.random.default_rng(4)
    qs, outs, tickets = [], [], []
    for k in range(80):
        gi = k % 2
        kind = "bfs" if k % 3 else "sssp"
        src = int(rng.integers(0, graphs[gi].n))
        out = serving.PinnedBuffer(graphs[gi].n, np.uint32 if kind == "bfs" else np.float32)
        qs.append((gi, kind, src))
        outs.append(out)
        tickets.append(srv.submit(gids[gi], kind, src, out))
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert all(r["status"] == 0 for r in res)
    assert st["workspace_bytes"] == before and st["evictions"] == 0
    for (gi, kind, src), out in zip(qs, outs):
        assert np.array_equal(out.array.view(np.uint32), _alone(sg, Gs[gi], kind, src, 0.1).view(np.uint32))
    small = serving.Server(slots=2, memory_budget=1 << 20)
    gid = small.add_graph(Gs[1])
    with pytest.raises(sg._lib.SygraphError):
        small.prepare(gid)
    assert small.stats()["evictions"] == 0
    small.close()
