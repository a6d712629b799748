"""The CPU model of the near-far schedule (tests/bucket_model.py) against the
oracle's Dijkstra, and the invariants of the work it counts."""
import numpy as np
import pytest

from bucket_model import near_far_model


@pytest.mark.parametrize("delta", [0.02, 0.0707, 0.1, 0.5, 4.0])
def test_model_distances_and_work(oracle, delta):
    g = oracle.rmat(12, 16, seed=1, weight_seed=2, perm_seed=3, value_type=1)
    deg = np.diff(np.asarray(g.row_offsets, np.int64))
    for src in [int(np.argmax(deg))] + [int(x) for x in oracle.sample_sources(g, 2, seed=5)]:
        d, buckets = near_far_model(g, src, delta)
        assert np.array_equal(d.view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32)), (delta, src)
        # every member is expanded at least once; members of different
        # buckets are distinct, so their heavy edges sum to at most m
        assert all(b["light_relaxations"] >= b["member_light_edges"] for b in buckets)
        assert sum(b["heavy_edges"] + b["member_light_edges"] for b in buckets) <= g.m
        assert sum(b["members"] for b in buckets) == int(np.sum(d < g.n + 1))
        assert [b["threshold"] for b in buckets] == sorted(b["threshold"] for b in buckets)
