"""Delta-stepping (sg_sssp_set_delta) and pull iterations (sg_sssp_set_pull):
every bucket width and direction rule gives the oracle's distances bit for
bit, since they only reorder relaxations towards the same least fixed point."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("delta", [0.01, 0.1, 0.5, 3.0, 1e6])
def test_nearfar_rmat_f32(sg, oracle, rmat, delta):
    g = rmat(14, perm_seed=3)
    G = sg.graph.build.fromCSR(g)
    s = sg.algorithms.SSSP(G)
    s.set_delta(delta)
    for src in [int(np.argmax(g.degrees()))] + [int(x) for x in sg.io.sample_sources(g, 2, seed=4)]:
        s.init(src)
        s.run()
        ref = oracle.sssp_dijkstra(g, src)
        assert np.array_equal(s.getDistances().view(np.uint32), ref.view(np.uint32)), (delta, src)


@pytest.mark.parametrize("delta", [1, 7, 64, 1000])
def test_nearfar_u32_grid_and_unreachable(sg, oracle, delta):
    g = sg.io.grid(80, 0.02, seed=1, weight_seed=2, value_type=sg.WEIGHT_U32)
    G = sg.graph.build.fromCSR(g)
    s = sg.algorithms.SSSP(G)
    s.set_delta(delta)
    for src in (0, 3200):
        s.init(src)
        s.run()
        assert np.array_equal(s.getDistances(), oracle.sssp_dijkstra(g, src))
    rng = np.random.default_rng(3)
    n = 2000
    w = (rng.integers(1, 1 << 24, 6000) / float(1 << 24)).astype(np.float32)
    gd = sg.io.fromCOO(n, rng.integers(0, n, 6000), rng.integers(0, n, 6000), w, dedupe=True,
                       drop_self_loops=True)
    s2 = sg.algorithms.SSSP(sg.graph.build.fromCSR(gd, sg.Properties(directed=True, weighted=True)))
    s2.set_delta(0.05)
    s2.init(7)
    s2.run()
    assert np.array_equal(s2.getDistances(), oracle.sssp_dijkstra(gd, 7))


@pytest.mark.parametrize("tail", [0.0, 1 / 64, 0.25, 1.0])
@pytest.mark.parametrize("delta", [0.02, 0.1])
def test_nearfar_bellman_ford_tail(sg, oracle, rmat, delta, tail):
    """Finishing with plain Bellman-Ford once the far set is small (any
    fraction, including 1: as soon as half the vertices are settled) keeps
    the distances; the log shows the buckets' heavy phases (push 4, pull 6)
    and refills (5)."""
    g = rmat(14, perm_seed=5)
    s = sg.algorithms.SSSP(sg.graph.build.fromCSR(g))
    s.set_delta(delta)
    s.set_tail(tail)
    for src in [int(x) for x in sg.io.sample_sources(g, 3, seed=6)]:
        s.init(src)
        it = s.run()
        assert np.array_equal(s.getDistances().view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32))
        kinds = [r["strategy"] for r in s.level_records()]
        assert kinds.count(0) + kinds.count(2) == it and (4 in kinds or 6 in kinds) and 5 in kinds
    gg = sg.io.grid(64, 0.02, seed=2, weight_seed=3, value_type=sg.WEIGHT_U32)
    s2 = sg.algorithms.SSSP(sg.graph.build.fromCSR(gg))
    s2.set_delta(int(delta * 640))
    s2.set_tail(tail)
    s2.init(100)
    s2.run()
    assert np.array_equal(s2.getDistances(), oracle.sssp_dijkstra(gg, 100))


@pytest.mark.parametrize("delta", [0.0, 0.05, 0.1])
def test_push_step_counts_in_the_log(sg, oracle, rmat, delta):
    """A push step's next_size against the frontier the next step expands:
    equal in the frontier Bellman-Ford (each newly set bit counted once), an
    upper bound in delta-stepping's push steps (marks are counted without
    waiting for the old bitmap word), and zero only where the run of push
    steps ends.  A refill's count is the next step's frontier exactly."""
    g = rmat(14, perm_seed=3)
    s = sg.algorithms.SSSP(sg.graph.build.fromCSR(g))
    s.set_delta(delta)
    for src in [int(np.argmax(g.degrees()))] + [int(x) for x in sg.io.sample_sources(g, 2, seed=8)]:
        s.init(src)
        it = s.run()
        assert np.array_equal(s.getDistances().view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32))
        recs = s.level_records()
        assert 0 < len(recs) < 4096 and sum(r["strategy"] == 0 for r in recs) == it
        assert recs[0]["strategy"] == 0 and recs[0]["frontier_size"] == 1
        for a, b in zip(recs, recs[1:]):
            if a["strategy"] == 0 and b["strategy"] == 0:
                assert a["next_size"] >= b["frontier_size"] > 0, (delta, src, a, b)
                if delta == 0.0:
                    assert a["next_size"] == b["frontier_size"], (src, a, b)
            if a["strategy"] == 0 and a["next_size"] == 0:
                assert b["strategy"] != 0, (delta, src, a, b)
            if a["strategy"] == 5 and b["strategy"] == 0:
                assert a["frontier_size"] == b["frontier_size"], (delta, src, a, b)
        assert recs[-1]["next_size"] == 0 or recs[-1]["strategy"] == 5


@pytest.mark.parametrize("light", [0, 16, 1 << 30])
@pytest.mark.parametrize("ratio", [0, 1, 8, 1 << 30])
def test_nearfar_heavy_pull(sg, oracle, rmat, ratio, light):
    """Heavy phases by pull (a bucket pulls when its heavy edges number more
    than m / ratio: never at 0, every bucket with a heavy edge at 2^30) or by
    push, and light iterations by pull (frontier above n / light) or push,
    give the oracle's distances; graphs with asymmetric weights stay on
    push."""
    g = rmat(15, perm_seed=7)
    s = sg.algorithms.SSSP(sg.graph.build.fromCSR(g))
    s.set_heavy_pull(ratio)
    s.set_light_pull(light)
    for delta in (0.03, 0.2):
        s.set_delta(delta)
        for src in [int(x) for x in sg.io.sample_sources(g, 2, seed=8)]:
            s.init(src)
            s.run()
            assert np.array_equal(s.getDistances().view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32))
            kinds = {r["strategy"] for r in s.level_records()}
            if ratio == 1 << 30:  # any bucket with a heavy edge pulls
                assert 6 in kinds
            if ratio == 0:
                assert 6 not in kinds
            if light == 1 << 30:  # every bucket iteration pulls
                assert 2 in kinds
            if light == 0:
                assert 2 not in kinds
    gg = sg.io.grid(64, 0.02, seed=4, weight_seed=5, value_type=sg.WEIGHT_U32)
    s2 = sg.algorithms.SSSP(sg.graph.build.fromCSR(gg))
    s2.set_heavy_pull(ratio)
    s2.set_light_pull(light)
    s2.set_delta(16)
    s2.init(77)
    s2.run()
    assert np.array_equal(s2.getDistances(), oracle.sssp_dijkstra(gg, 77))
    # asymmetric weights on an undirected-looking edge set: pull must not run
    rng = np.random.default_rng(9)
    n = 3000
    a = rng.integers(0, n, 20000)
    b = rng.integers(0, n, 20000)
    w = (rng.integers(1, 1 << 24, 40000) / float(1 << 24)).astype(np.float32)
    ga = sg.io.fromCOO(n, np.concatenate([a, b]), np.concatenate([b, a]), w, dedupe=True, drop_self_loops=True)
    s3 = sg.algorithms.SSSP(sg.graph.build.fromCSR(ga, sg.Properties(directed=True, weighted=True)))
    s3.set_heavy_pull(1 << 30)
    s3.set_light_pull(1 << 30)
    s3.set_delta(0.05)
    s3.init(1)
    s3.run()
    assert np.array_equal(s3.getDistances().view(np.uint32), oracle.sssp_dijkstra(ga, 1).view(np.uint32))
    assert not {2, 6} & {r["strategy"] for r in s3.level_records()}


def test_nearfar_argument_checks_and_reset(sg, oracle, rmat):
    g = rmat(10)
    s = sg.algorithms.SSSP(sg.graph.build.fromCSR(g))
    with pytest.raises(sg._lib.SygraphError):
        s.set_delta(-1.0)
    for bad in (-0.1, 1.5):
        with pytest.raises(sg._lib.SygraphError):
            s.set_tail(bad)
    s.set_delta(0.2)
    s.init(3)
    s.run()
    a = s.getDistances()
    s.set_delta(0.0)  # back to the reference schedule
    s.init(3)
    s.run()
    assert np.array_equal(a.view(np.uint32), s.getDistances().view(np.uint32))


def test_instances_on_own_streams_with_grid_caps(sg, oracle, rmat):
    """Two instances on separate streams with a share of the SMs each, run
    back to back without a host wait, give the single-instance results."""
    import ctypes as C
    g = rmat(13, perm_seed=2)
    G = sg.graph.build.fromCSR(g)
    streams = []
    for _ in range(2):
        h = C.c_void_p()
        sg._lib.call("sg_stream_create", C.byref(h))
        streams.append(h)
    b = sg.algorithms.BFS(G)
    s = sg.algorithms.SSSP(G)
    sg._lib.call("sg_bfs_set_launch", b.handle, streams[0], 74)
    sg._lib.call("sg_sssp_set_launch", s.handle, streams[1], 74)
    s.set_delta(0.3)
    src = int(np.argmax(g.degrees()))
    b.init(src)
    s.init(src)
    b.run_async(2, 15.0, 24.0)
    s.run_async()
    assert np.array_equal(b.getDistances(), oracle.bfs_levels(g, src))
    assert np.array_equal(s.getDistances().view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32))
    # an instance uses its stream until it is destroyed: destroy the instances first
    del b, s
    import gc
    gc.collect()
    for h in streams:
        sg._lib.call("sg_stream_destroy", h)


@pytest.mark.parametrize("ratio", [1, 4, 1000])
@pytest.mark.parametrize("delta", [0.0, 0.1])
def test_pull_iterations_rmat_f32(sg, oracle, rmat, ratio, delta):
    g = rmat(14, perm_seed=3)
    s = sg.algorithms.SSSP(sg.graph.build.fromCSR(g))
    s.set_pull(ratio)
    s.set_delta(delta)
    for src in [int(np.argmax(g.degrees()))] + [int(x) for x in sg.io.sample_sources(g, 2, seed=4)]:
        s.init(src)
        s.run()
        ref = oracle.sssp_dijkstra(g, src)
        assert np.array_equal(s.getDistances().view(np.uint32), ref.view(np.uint32)), (ratio, delta, src)
    if ratio == 1000 and delta == 0.0:  # pull iterations run without buckets only
        assert any(r["strategy"] == 2 for r in s.level_records())


def test_pull_iterations_directed_hubs_and_u32(sg, oracle):
    rng = np.random.default_rng(8)
    n = 6000
    hubs = rng.integers(0, n, 5)
    src = np.concatenate([rng.integers(0, n, 40000), rng.integers(0, n, 8000)])
    dst = np.concatenate([rng.integers(0, n, 40000), np.repeat(hubs, 1600)])  # hubs: in-degree > 256
    w = (rng.integers(1, 1 << 24, src.size) / float(1 << 24)).astype(np.float32)
    gd = sg.io.fromCOO(n, src, dst, w, dedupe=True, drop_self_loops=True)
    s = sg.algorithms.SSSP(sg.graph.build.fromCSR(gd, sg.Properties(directed=True, weighted=True)))
    for ratio, delta in ((1000, 0.0), (1000, 0.05), (2, 0.0)):
        s.set_pull(ratio)
        s.set_delta(delta)
        for v in (int(hubs[0]), 11):
            s.init(v)
            s.run()
            assert np.array_equal(s.getDistances(), oracle.sssp_dijkstra(gd, v)), (ratio, delta, v)
    gg = sg.io.grid(80, 0.02, seed=1, weight_seed=2, value_type=sg.WEIGHT_U32)
    s2 = sg.algorithms.SSSP(sg.graph.build.fromCSR(gg))
    s2.set_pull(1000)
    s2.set_delta(64)
    s2.init(0)
    s2.run()
    assert np.array_equal(s2.getDistances(), oracle.sssp_dijkstra(gg, 0))


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


@pytest.mark.parametrize("delta", [0.02, 0.1])
def test_learned_heavy_phases(sg, oracle, rmat, delta):
    """The learned heavy phase (sg_sssp_set_selector) keeps the oracle's
    distances; at every heavy phase the device takes the MLP's choice between
    push (4) and pull (6) on the logged features; without a model the
    heavy_pull rule decides, and its forced forms give the same features."""
    from sygraph_b200 import selector
    g = rmat(14, perm_seed=3)
    G = sg.graph.build.fromCSR(g)
    assert G.weight_sorted()[2]  # symmetric weighted rows: pull is possible
    s = sg.algorithms.SSSP(G)
    s.set_delta(delta)
    s.log_features(True)
    srcs = [int(np.argmax(g.degrees()))] + [int(x) for x in sg.io.sample_sources(g, 2, seed=4)]
    phases = 0
    for seed in range(3):
        m = _trusting_mlp(selector, seed)
        s.set_selector(m, margin=0.0)
        for src in srcs:
            s.init(src)
            s.run()
            ref = oracle.sssp_dijkstra(g, src)
            assert np.array_equal(s.getDistances().view(np.uint32), ref.view(np.uint32)), (seed, src)
            got = np.array([2 if r["strategy"] == 6 else 0 for r in s.level_records() if r["strategy"] in (4, 6)])
            F = s.level_features()
            assert len(F) == len(got) and np.all(np.isfinite(F))
            if not len(F):
                continue
            y = m.forward(F)[:, [0, 2]]
            pick = np.where(got == 2, 1, 0)
            best = y.min(1)
            assert np.all(y[np.arange(len(got)), pick] <= best + 1e-4 * (1 + np.abs(best))), (seed, src)
            phases += len(F)
    assert phases >= 6
    s.set_selector(None)
    # without a model: the rule (pull when the bucket's heavy edges exceed
    # m / ratio, feature 3 = heavy edges / m) and its forced forms
    src = srcs[0]
    for ratio in (0, 8, 0xFFFFFFFF):
        s.set_heavy_pull(ratio)
        s.init(src)
        s.run()
        assert np.array_equal(s.getDistances().view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32))
        F = s.level_features()
        got = np.array([2 if r["strategy"] == 6 else 0 for r in s.level_records() if r["strategy"] in (4, 6)])
        assert len(F) == len(got) and len(F) >= 2
        if ratio == 0:
            assert np.all(got == 0)
        elif ratio == 8:
            clear = np.abs(F[:, 3] * 8 - 1) > 1e-3
            assert np.array_equal(got[clear], np.where(F[clear, 3] * 8 > 1, 2, 0))
        else:
            assert np.all(got[F[:, 3] > 0] == 2)
    s.set_heavy_pull(8)
    s.log_features(False)
