"""The autotuner's host logic (no GPU): it keeps the fastest candidate,
caches it per key and honours the cache; candidate lists."""
import json

from sygraph_b200 import autotune


def test_tune_picks_fastest_and_caches(tmp_path):
    cost = {1: 0.003, 2: 0.001, 3: 0.002}
    calls = []

    def run(c):
        calls.append(c)
        # deterministic fake work: spin for the candidate's cost
        import time
        t = time.perf_counter()
        while time.perf_counter() - t < cost[c]:
            pass

    path = tmp_path / "tune.json"
    pick, timings = autotune.tune("k", [1, 2, 3], run, reps=2, path=path)
    assert pick == 2 and len(timings) == 3
    assert json.loads(path.read_text())["k"] == 2
    calls.clear()
    pick2, t2 = autotune.tune("k", [1, 2, 3], run, reps=2, path=path)
    assert pick2 == 2 and t2 == {} and not calls  # served from the cache
    # a cached value that is no longer a candidate is re-tuned
    pick3, _ = autotune.tune("k", [1, 3], run, reps=1, path=path)
    assert pick3 == 3


def test_delta_candidates():
    f = autotune.delta_candidates(0.5, integer=False)
    assert len(f) == 15 and abs(f[0] - 0.05) < 1e-12 and abs(f[-1] - 6.4) < 1e-9
    assert all(abs(b / a - 2 ** 0.5) < 1e-9 for a, b in zip(f, f[1:]))
    u = autotune.delta_candidates(32.5, integer=True)
    assert u == sorted(set(u)) and u[0] >= 1 and all(float(x).is_integer() for x in u)


import numpy as np  # noqa: E402
import pytest  # noqa: E402


@pytest.mark.gpu
def test_tuned_engines_keep_their_results(sg, oracle, rmat, tmp_path, monkeypatch):
    monkeypatch.setenv("SYGRAPH_B200_TUNE_CACHE", str(tmp_path / "t.json"))
    g = rmat(13, perm_seed=4)
    G = sg.graph.build.fromCSR(g)
    srcs = sg.io.sample_sources(g, 16, seed=2)
    mb = sg.algorithms.MultiBFS(G, 64)
    pick = autotune.tune_batched_bfs(mb, srcs, reps=1)
    assert pick["max_ctas"] in autotune.grid_candidates()
    mb.run(srcs, 2, pick["alpha"], 24.0)
    assert np.array_equal(mb.getDistances(), oracle.bfs_multi(g, srcs))
    bc = sg.algorithms.BatchedBC(G)
    autotune.tune_batched_bc(bc, srcs, reps=1)
    bc.run(srcs)
    ref = oracle.bc(g, srcs)
    np.testing.assert_allclose(bc.getBC(), ref, rtol=1e-4, atol=1e-4 * max(1.0, float(ref.max())) * 1e-3)
    sp = sg.algorithms.SSSP(G)
    d = autotune.tune_sssp(sp, srcs[:2], autotune.mean_weight(g), reps=1)["delta"]
    assert d >= 0.0
    sp.init(int(srcs[0]))
    sp.run()
    assert np.array_equal(sp.getDistances().view(np.uint32), oracle.sssp_dijkstra(g, int(srcs[0])).view(np.uint32))
    assert json.loads((tmp_path / "t.json").read_text())  # choices were cached
