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


def _trusting_mlp(selector, seed):
    """A random MLP whose trusted range covers every feature value."""
    rng = np.random.default_rng(seed)
    m = selector.Mlp()
    p = m.params
    t, I = selector.TRAINABLE_COUNT, selector.IN
    p[:t] = rng.normal(scale=0.5, size=t).astype(np.float32)
    p[t:t + I] = 0.0
    p[t + I:t + 2 * I] = 1.0
    p[t + 2 * I:t + 3 * I] = -1e9
    p[t + 3 * I:t + 4 * I] = 1e9
    m.params = p
    return m


def _batched_heuristic(recs, n, alpha, beta):
    """The batched engine's heuristic choice (0 push, 2 pull) for every level
    after the first, given the direction each level actually took."""
    f32 = np.float32
    out = [0]
    for r in recs[:-1]:
        if r["strategy"] < 2:
            pull = f32(r["next_degree"]) > f32(r["unexplored_degree"]) / f32(alpha)
        else:
            pull = not f32(r["next_size"]) < f32(n) / f32(beta)
        out.append(2 if pull else 0)
    return np.array(out)


@pytest.mark.parametrize("scale,perm", [(12, 0), (15, 3)])
def test_msbfs_forced_and_learned_schedules_keep_depths(sg, oracle, rmat, scale, perm):
    """Forced per-level directions and the learned mode change the work, not
    the depths; the learned mode asks the model where the heuristic switches
    direction and takes its argmin over push and pull there, the heuristic's
    choice elsewhere; the feature log covers every level."""
    from sygraph_b200 import selector
    g = rmat(scale, perm_seed=perm)
    G = sg.graph.build.fromCSR(g)
    srcs = sg.io.sample_sources(g, 64, seed=5)
    ref = oracle.bfs_multi(g, srcs)
    mb = sg.algorithms.MultiBFS(G, 64)
    rng = np.random.default_rng(scale)
    for _ in range(3):
        sched = rng.choice([0, 2], size=32)
        mb.set_schedule(sched)
        mb.run(srcs, 2, 4.0, 24.0)
        assert np.array_equal(mb.getDistances(), ref)
        got = [r["strategy"] for r in mb.level_records()]
        assert got == list(sched[:len(got)])
    mb.set_schedule([])
    with pytest.raises(sg._lib.SygraphError):
        mb.set_schedule([1])
    with pytest.raises(sg._lib.SygraphError):
        mb.run(srcs, sg.algorithms.bfs_direction.learned, 4.0, 24.0)  # no selector yet
    asked = 0
    for seed in range(4):
        m = _trusting_mlp(selector, seed)
        mb.set_selector(m, margin=0.0)
        mb.log_features(True)
        det = mb.run(srcs, sg.algorithms.bfs_direction.learned, 4.0, 24.0)
        assert np.array_equal(mb.getDistances(), ref)
        recs = mb.level_records()
        F = mb.level_features()
        assert F.shape == (det["iterations"], 12) and np.all(np.isfinite(F))
        got = np.array([r["strategy"] for r in recs])
        assert set(np.unique(got)) <= {0, 2}
        heur = _batched_heuristic(recs, g.n, 4.0, 24.0)
        cur = np.concatenate([[0], got[:-1]])
        ask = (heur >= 2) != (cur >= 2)
        assert np.array_equal(got[~ask], heur[~ask])
        y = m.forward(F)[:, [0, 2]]
        pick = np.where(got == 2, 1, 0)
        best = y.min(1)
        ok = y[np.arange(len(got)), pick] <= best + 1e-4 * (1 + np.abs(best))
        assert np.all(ok[ask])
        asked += int(ask.sum())
    assert asked >= 2
    mb.set_selector(None)
    mb.log_features(False)
