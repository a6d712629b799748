"""The six per-level BFS strategies (push / pull / pull_all, each warp- or
CTA-mapped), forced schedules and the learned selector: every schedule must
give the oracle's depths bit for bit, since BFS levels are unique and only
the work mapping changes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STRATS = range(6)


def _graphs(sg, rmat):
    n = 5000
    path = sg.io.fromCOO(n, np.arange(n - 1), np.arange(1, n), symmetrize=True)
    star_n = 70_000
    star = sg.io.fromCOO(star_n, np.zeros(star_n - 1, np.uint32), np.arange(1, star_n, dtype=np.uint32),
                         symmetrize=True)
    return {"rmat14": rmat(14, perm_seed=7), "grid": sg.io.grid(96), "path": path, "star": star}


@pytest.fixture(scope="module")
def graphs(sg, rmat):
    return _graphs(sg, rmat)


def _sources(sg, g):
    return [int(np.argmax(g.degrees()))] + [int(s) for s in sg.io.sample_sources(g, 2, seed=11)]


@pytest.mark.parametrize("name", ["rmat14", "grid", "path", "star"])
@pytest.mark.parametrize("strategy", STRATS)
def test_forced_strategy_parity(sg, oracle, graphs, name, strategy):
    g = graphs[name]
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    bfs.set_schedule([strategy] * 8192)
    for s in _sources(sg, g):
        bfs.init(s)
        det = bfs.run(sg.algorithms.bfs_direction.hybrid, 15.0, 24.0)
        ref = oracle.bfs_levels(g, s)
        assert np.array_equal(bfs.getDistances(), ref), (name, strategy, s)
        recs = bfs.level_records()
        assert all(r["strategy"] == strategy for r in recs)
        assert det.visited_vertices == int((ref != g.n + 1).sum())
        assert det.visited_edges == oracle.visited_edges(g, ref, g.n + 1)


def test_random_schedules(sg, oracle, graphs):
    rng = np.random.default_rng(5)
    for name in ("rmat14", "grid", "star"):
        g = graphs[name]
        G = sg.graph.build.fromCSR(g)
        bfs = sg.algorithms.BFS(G)
        for s in _sources(sg, g):
            sched = rng.integers(-1, 6, size=64).astype(np.int32)
            bfs.set_schedule(sched)
            bfs.init(s)
            bfs.run(sg.algorithms.bfs_direction.push)
            assert np.array_equal(bfs.getDistances(), oracle.bfs_levels(g, s))
            recs = bfs.level_records()
            for r in recs:
                want = sched[r["level"]] if r["level"] < len(sched) else -1
                # unscheduled levels: push mode always decides push/warp
                assert r["strategy"] == (want if want >= 0 else 0)
        bfs.set_schedule(None)


def test_directed_graph_forced_pull(sg, oracle):
    rng = np.random.default_rng(5)
    n = 3000
    g = sg.io.fromCOO(n, rng.integers(0, n, 20000), rng.integers(0, n, 20000), dedupe=True, drop_self_loops=True)
    G = sg.graph.build.fromCSR(g, sg.Properties(directed=True))
    bfs = sg.algorithms.BFS(G)
    s0 = int(np.argmax(g.degrees()))
    for strategy in STRATS:
        bfs.set_schedule([strategy] * 64)
        bfs.init(s0)
        bfs.run(2, 2.0, 4.0)
        ref, _, _ = oracle.bfs_frontier(g, s0, 0, 1.0, 1.0)
        assert np.array_equal(bfs.getDistances(), ref)


def test_schedule_argument_checks(sg, graphs):
    G = sg.graph.build.fromCSR(graphs["grid"])
    bfs = sg.algorithms.BFS(G)
    with pytest.raises(sg._lib.SygraphError):
        bfs.set_schedule([0, 6])
    with pytest.raises(sg._lib.SygraphError):
        bfs.set_schedule([-2])
    bfs.init(0)
    with pytest.raises(sg._lib.SygraphError) as ei:
        bfs.run(sg.algorithms.bfs_direction.learned)  # no selector attached
    assert ei.value.status == sg._lib.SG_ERR_NOT_INITIALIZED


def _trusting_mlp(selector, seed):
    """A random MLP whose trusted range covers every feature value."""
    rng = np.random.default_rng(seed)
    m = selector.Mlp()
    p = m.params
    t = selector.TRAINABLE_COUNT
    p[:t] = rng.normal(scale=0.5, size=t).astype(np.float32)
    I = selector.IN
    p[t:t + I] = 0.0
    p[t + I:t + 2 * I] = 1.0
    p[t + 2 * I:t + 3 * I] = -1e9
    p[t + 3 * I:t + 4 * I] = 1e9
    m.params = p
    return m


def _heuristic_levels(recs, n, alpha, beta):
    """The reference heuristic's choice (0 push, 2 pull) for every level, from
    the level records of the run and the strategy each level actually took,
    in the engine's float arithmetic (bfs.hpp:325-350)."""
    f32 = np.float32
    out = [0]  # level 0 starts in push
    for prev in recs[:-1]:
        if prev["strategy"] < 2:
            pull = f32(np.uint32(prev["next_degree"] & 0xFFFFFFFF)) > \
                f32(np.uint32(prev["unexplored_degree"] & 0xFFFFFFFF)) / f32(alpha)
        else:
            pull = not f32(prev["next_size"]) < f32(n) / f32(beta)
        out.append(2 if pull else 0)
    return out


def test_learned_mode_parity_and_mask(sg, oracle, graphs):
    """The model is asked where the heuristic switches direction and where
    the heuristic's choice is not allowed; there the device takes the MLP's
    argmin over the allowed strategies, elsewhere the heuristic's choice."""
    from sygraph_b200 import selector
    asked = 0
    for name in ("rmat14", "grid", "star"):
        g = graphs[name]
        G = sg.graph.build.fromCSR(g)
        bfs = sg.algorithms.BFS(G)
        for seed, allowed in ((1, 0x3F), (2, 0x03), (3, 0x0C), (4, 0x30), (5, 0x21)):
            m = _trusting_mlp(selector, seed)
            bfs.set_selector(m, allowed, margin=0.0, min_frontier=0.0)  # plain argmin where asked
            bfs.log_features(True)
            for s in _sources(sg, g)[:2]:
                bfs.init(s)
                det = bfs.run(sg.algorithms.bfs_direction.learned, 15.0, 24.0)
                assert np.array_equal(bfs.getDistances(), oracle.bfs_levels(g, s)), (name, seed, s)
                recs = bfs.level_records()
                assert all((allowed >> r["strategy"]) & 1 for r in recs)
                F = bfs.level_features()
                assert F.shape == (det.iterations, 12) and np.all(np.isfinite(F))
                got = np.array([r["strategy"] for r in recs])
                heur = np.array(_heuristic_levels(recs, g.n, 15.0, 24.0))
                cur = np.concatenate([[0], got[:-1]])
                ask = np.array([(h >= 2) != (c >= 2) or not (allowed >> int(h)) & 1 for h, c in zip(heur, cur)])
                assert np.array_equal(got[~ask], heur[~ask]), (name, seed, s)
                # where asked, the device's choice is the MLP's argmin on the
                # logged features (up to float summation order between the two
                # forward passes)
                y = m.forward(F)
                y[:, [j for j in range(6) if not (allowed >> j) & 1]] = np.inf
                best = y.min(1)
                ok = y[np.arange(len(got)), got] <= best + 1e-4 * (1 + np.abs(best))
                assert np.all(ok[ask]), (name, seed, s)
                asked += int(ask.sum())
    assert asked >= 30


def test_learned_mode_small_frontiers_keep_the_heuristic(sg, oracle, rmat):
    """Frontiers below min_frontier * n take the heuristic's choice without an
    inference (when it is allowed); 1.0 leaves every level to the heuristic."""
    from sygraph_b200 import selector
    g = rmat(14, perm_seed=7)
    bfs = sg.algorithms.BFS(sg.graph.build.fromCSR(g))
    s = int(np.argmax(g.degrees()))
    ref, it, steps = oracle.bfs_frontier(g, s, 2, 15.0, 24.0)
    bfs.set_selector(_trusting_mlp(selector, 9), margin=0.0, min_frontier=1.0)
    bfs.init(s)
    bfs.run(sg.algorithms.bfs_direction.learned, 15.0, 24.0)
    assert np.array_equal(bfs.getDistances(), ref)
    assert [r["strategy"] for r in bfs.level_records()] == [2 * x for x in steps]
    # restricted to pull_all: the heuristic's push / pull is not allowed, so the MLP decides
    bfs.set_selector(_trusting_mlp(selector, 9), allowed=0x30, margin=0.0, min_frontier=1.0)
    bfs.init(s)
    bfs.run(sg.algorithms.bfs_direction.learned, 15.0, 24.0)
    assert np.array_equal(bfs.getDistances(), ref)
    assert all(r["strategy"] in (4, 5) for r in bfs.level_records())
    with pytest.raises(sg._lib.SygraphError):
        bfs.set_selector(None, min_frontier=2.0)


def test_learned_mode_falls_back_to_heuristic_outside_range(sg, oracle, rmat):
    from sygraph_b200 import selector
    g = rmat(14, perm_seed=7)
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    m = selector.Mlp()
    p = m.params
    t, I = selector.TRAINABLE_COUNT, selector.IN
    p[t + 2 * I:t + 3 * I] = 1e9  # lo > every feature: nothing is trusted
    p[t + 3 * I:t + 4 * I] = 2e9
    m.params = p
    bfs.set_selector(m)
    s = int(np.argmax(g.degrees()))
    bfs.init(s)
    det = bfs.run(sg.algorithms.bfs_direction.learned, 15.0, 24.0)
    ref, it, steps = oracle.bfs_frontier(g, s, 2, 15.0, 24.0)
    assert np.array_equal(bfs.getDistances(), ref)
    assert det.iterations == it
    assert sorted(det.pull_steps) == [i for i, x in enumerate(steps) if x == 1]


def test_feature_log_matches_level_records(sg, rmat):
    g = rmat(12, perm_seed=0)
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    bfs.log_features(True)
    s = int(np.argmax(g.degrees()))
    bfs.init(s)
    det = bfs.run(sg.algorithms.bfs_direction.hybrid, 15.0, 24.0)
    F = bfs.level_features()
    recs = bfs.level_records()
    assert len(F) == det.iterations == len(recs)
    n = g.n
    for i, r in enumerate(recs):
        # feature 1: frontier size / n of the level the features choose for
        assert F[i, 1] == pytest.approx(r["frontier_size"] / n, rel=1e-5)
        # features 6, 7: bitmap / summary occupancy of a randomly spread frontier of that size
        w0 = (n + 31) // 32
        w1 = (w0 + 31) // 32
        assert F[i, 6] == pytest.approx(1 - np.exp(-r["frontier_size"] / w0), rel=1e-4, abs=1e-6)
        assert F[i, 7] == pytest.approx(1 - np.exp(-r["frontier_size"] / (32 * w1)), rel=1e-4, abs=1e-6)
        if i > 0:
            assert F[i, 10] == (1.0 if recs[i - 1]["strategy"] >= 2 else 0.0)


def test_learned_mode_margin_keeps_the_heuristic(sg, oracle, rmat):
    """A margin no prediction can clear leaves every level to the heuristic."""
    from sygraph_b200 import selector
    g = rmat(14, perm_seed=7)
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    bfs.set_selector(_trusting_mlp(selector, 9), margin=99.0)
    s = int(np.argmax(g.degrees()))
    bfs.init(s)
    det = bfs.run(sg.algorithms.bfs_direction.learned, 15.0, 24.0)
    ref, it, steps = oracle.bfs_frontier(g, s, 2, 15.0, 24.0)
    assert np.array_equal(bfs.getDistances(), ref) and det.iterations == it
    assert [r["strategy"] for r in bfs.level_records()] == [2 * x for x in steps]
    with pytest.raises(sg._lib.SygraphError):
        bfs.set_selector(None, margin=-1.0)
