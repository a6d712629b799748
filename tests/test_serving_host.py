"""Host side of serving (no GPU): the seeded open-loop workload and the
latency summary."""
import numpy as np


def test_workload_rate_mix_and_determinism(sg):
    from sygraph_b200 import serving
    sizes = [1 << 14, 1 << 16, 1 << 20]
    wl = serving.make_workload(sizes, qps=2000.0, duration_s=5.0, bfs_fraction=0.7, seed=3)
    n = wl.arrivals.size
    assert abs(n - 10000) < 4 * np.sqrt(10000)  # Poisson count
    assert np.all(np.diff(wl.arrivals) > 0) and wl.arrivals[-1] < 5.0
    frac = sum(k == "bfs" for k in wl.kind) / n
    assert abs(frac - 0.7) < 0.03
    assert all(s < sizes[g] for s, g in zip(wl.source, wl.graph))
    wl2 = serving.make_workload(sizes, qps=2000.0, duration_s=5.0, bfs_fraction=0.7, seed=3)
    assert np.array_equal(wl.arrivals, wl2.arrivals) and wl.kind == wl2.kind


def test_percentiles(sg):
    from sygraph_b200 import serving
    p = serving.percentiles(np.arange(1, 101, dtype=float))
    assert abs(p["p50_ms"] - 50.5) < 1e-9 and abs(p["p99_ms"] - 99.01) < 1e-9
    assert serving.percentiles([])["p50_ms"] is None
