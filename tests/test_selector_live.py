"""The learned selector timed live on the GPU against the reference
heuristic (bfs.hpp:325-350) on the evaluation graphs of the selector: RMAT-22
(the benchmark graph) and the 4096 x 4096 grid with 2% long-range pairs.
Both modes give identical depths (BFS levels are unique); the learned mode
must not lose on RMAT-22 and must win on the grid, inference cost included.

Timing: launches of the two modes alternate back to back on one stream,
each between two CUDA events, so both see the same clocks and caches; the
ratio is of the medians over every source and repetition."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

REPS = 12
HYBRID, LEARNED = 2, 3


def _timed_ratio(sg, g, sources):
    import torch
    from sygraph_b200 import selector
    G = sg.graph.build.fromCSR(g)
    h, l = sg.algorithms.BFS(G), sg.algorithms.BFS(G)
    l.set_selector(selector.Mlp.load())
    for s in sources:
        h.init(int(s))
        h.run(HYBRID, 15.0, 24.0)
        l.init(int(s))
        l.run(LEARNED, 15.0, 24.0)
        assert np.array_equal(h.getDistances(), l.getDistances()), int(s)
    th, tl = [], []
    for _ in range(REPS + 2):  # the first two rounds warm up
        pairs = []
        for s in sources:
            for inst, mode, out in ((h, HYBRID, th), (l, LEARNED, tl)):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                inst.init(int(s))
                a.record()
                inst.run_async(mode, 15.0, 24.0)
                b.record()
                pairs.append((a, b, out))
        torch.cuda.synchronize()
        for a, b, out in pairs:
            out.append(a.elapsed_time(b))
    th, tl = th[2 * len(sources):], tl[2 * len(sources):]
    return float(np.median(th)) / float(np.median(tl))


def test_learned_no_slower_on_rmat22(sg):
    g = sg.io.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, weight_seed=2, perm_seed=0, value_type=sg.WEIGHT_F32)
    ratio = _timed_ratio(sg, g, sg.io.sample_sources(g, 8, seed=3))
    assert ratio >= 0.99, ratio


def test_learned_faster_on_grid4096(sg):
    g = sg.io.grid(4096, long_range_frac=0.02, seed=103, weight_seed=2, value_type=sg.WEIGHT_U32)
    ratio = _timed_ratio(sg, g, sg.io.sample_sources(g, 4, seed=3))
    assert ratio >= 1.10, ratio
