"""The learned selector timed live on the GPU against the reference
heuristic (bfs.hpp:325-350) on the evaluation graphs of the selector: RMAT-22
(the benchmark graph) and the 4096 x 4096 grid with 2% long-range pairs.
Both modes give identical depths (BFS levels are unique); the learned mode
must not lose on RMAT-22 and must win on the grid, inference cost included.

Timing: one instance with the model attached runs both modes (the same
buffers, so memory placement cannot favour either), the two launches of a
source back to back on one stream between CUDA events, in alternating order
from one repetition to the next.  Each source's time is its median over the
repetitions; the ratio is of the sums over the sources (the time to traverse
them all), so every source weighs by its length."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

REPS = 12
HYBRID, LEARNED = 2, 3


def _alternating(torch, launch, keys, reps=REPS, warm=2):
    """Median event time per key of launch(key, start, end), the keys' order
    reversed every other repetition; the first `warm` repetitions are
    dropped."""
    t = {k: [] for k in keys}
    for rep in range(reps + warm):
        pairs = []
        for k in (keys if rep % 2 == 0 else keys[::-1]):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            launch(k, a, b)
            pairs.append((k, a, b))
        torch.cuda.synchronize()
        if rep >= warm:
            for k, a, b in pairs:
                t[k].append(a.elapsed_time(b))
    return {k: float(np.median(v)) for k, v in t.items()}


def _timed_ratio(sg, g, sources):
    import torch
    from sygraph_b200 import selector
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    bfs.set_selector(selector.Mlp.load())
    for s in sources:
        bfs.init(int(s))
        bfs.run(HYBRID, 15.0, 24.0)
        ref = bfs.getDistances()
        bfs.init(int(s))
        bfs.run(LEARNED, 15.0, 24.0)
        assert np.array_equal(ref, bfs.getDistances()), int(s)

    def launch(key, a, b):
        s, mode = key
        bfs.init(int(s))
        a.record()
        bfs.run_async(mode, 15.0, 24.0)
        b.record()

    th = tl = 0.0
    for s in sources:
        m = _alternating(torch, launch, [(s, HYBRID), (s, LEARNED)])
        th += m[(s, HYBRID)]
        tl += m[(s, LEARNED)]
    return th / tl


def test_learned_no_slower_on_rmat22(sg):
    g = sg.io.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, weight_seed=2, perm_seed=0, value_type=sg.WEIGHT_F32)
    ratio = _timed_ratio(sg, g, sg.io.sample_sources(g, 16, seed=3))
    assert ratio >= 0.99, ratio


def test_learned_faster_on_grid4096(sg):
    g = sg.io.grid(4096, long_range_frac=0.02, seed=103, weight_seed=2, value_type=sg.WEIGHT_U32)
    ratio = _timed_ratio(sg, g, sg.io.sample_sources(g, 4, seed=3))
    assert ratio >= 1.10, ratio


def _batched_ratio(sg, g, alpha):
    """Heuristic / learned launch time of the batched BFS (64 sources), both
    modes on one instance alternating on one stream; identical depths."""
    import torch
    from sygraph_b200 import selector, train_selector
    G = sg.graph.build.fromCSR(g)
    srcs = sg.io.sample_sources(g, 64, seed=3)
    mb = sg.algorithms.MultiBFS(G, 64)
    mb.set_selector(selector.Mlp.load(train_selector.BATCHED_MODEL_PATH))
    mb.run(srcs, HYBRID, alpha, 24.0)
    ref = mb.getDistances()
    mb.run(srcs, LEARNED, alpha, 24.0)
    assert np.array_equal(ref, mb.getDistances())

    def launch(mode, a, b):
        a.record()
        mb.run_async(srcs, mode, alpha, 24.0)
        b.record()

    m = _alternating(torch, launch, [HYBRID, LEARNED])
    return m[HYBRID] / m[LEARNED]


def test_learned_batched_no_slower_on_rmat22(sg):
    g = sg.io.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, weight_seed=2, perm_seed=0, value_type=sg.WEIGHT_F32)
    ratio = _batched_ratio(sg, g, 4.0)
    assert ratio >= 0.99, ratio


def test_learned_batched_faster_on_grid4096(sg):
    g = sg.io.grid(4096, long_range_frac=0.02, seed=103, weight_seed=2, value_type=sg.WEIGHT_U32)
    ratio = _batched_ratio(sg, g, 4.0)
    assert ratio >= 1.02, ratio


def _sssp_ratio(sg, g, sources, delta):
    """Rule / learned time of delta-stepping SSSP (heavy phases chosen by the
    SSSP model), both on one instance alternating on one stream, per-source
    medians summed; identical distances."""
    import torch
    from sygraph_b200 import selector, train_selector
    G = sg.graph.build.fromCSR(g)
    sp = sg.algorithms.SSSP(G)
    sp.set_delta(delta)
    mdl = selector.Mlp.load(train_selector.SSSP_MODEL_PATH)
    for s in sources:
        sp.set_selector(None)
        sp.init(int(s))
        sp.run()
        ref = sp.getDistances().view(np.uint32).copy()
        sp.set_selector(mdl)
        sp.init(int(s))
        sp.run()
        assert np.array_equal(ref, sp.getDistances().view(np.uint32)), int(s)

    def launch(key, a, b):
        s, learned = key
        sp.set_selector(mdl if learned else None)
        sp.init(int(s))
        a.record()
        sp.run_async()
        b.record()

    th = tl = 0.0
    for s in sources:
        m = _alternating(torch, launch, [(s, False), (s, True)], reps=6)
        th += m[(s, False)]
        tl += m[(s, True)]
    return th / tl


def test_learned_sssp_no_slower_on_rmat22(sg):
    g = sg.io.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, weight_seed=2, perm_seed=0, value_type=sg.WEIGHT_F32)
    assert _sssp_ratio(sg, g, sg.io.sample_sources(g, 4, seed=3), 0.1) >= 0.99


def test_learned_sssp_no_slower_on_uniform21(sg):
    g = sg.io.rmat(21, 16, 0.25, 0.25, 0.25, seed=104, weight_seed=2, value_type=sg.WEIGHT_F32)
    assert _sssp_ratio(sg, g, sg.io.sample_sources(g, 4, seed=3), 0.2) >= 0.99
