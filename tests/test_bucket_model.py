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


def test_pull_scan_count_against_a_row_by_row_walk(oracle):
    """The vectorised count of the heavy-phase pull's reads equals a plain
    walk of each candidate's weight-sorted row with the kernel's stop rule."""
    from bucket_model import pull_scan_edges, weight_sorted

    g = oracle.rmat(9, 8, seed=2, weight_seed=3, perm_seed=1, value_type=1)
    ro = np.asarray(g.row_offsets, np.int64)
    col_s, w_s = weight_sorted(ro, np.asarray(g.column_indices, np.int64), np.asarray(g.values, np.float32))
    n = len(ro) - 1
    assert all(np.all(np.diff(w_s[ro[v]:ro[v + 1]]) >= 0) for v in range(n))
    rng = np.random.default_rng(4)
    dist = rng.random(n).astype(np.float32) * 2
    dist[rng.random(n) < 0.3] = np.inf
    lo, thr = np.float32(0.3), np.float32(0.4)
    member = (dist >= lo) & (dist < thr)
    want, cands = 0, 0
    for v in range(n):
        if not dist[v] > thr:
            continue
        cands += 1
        best = dist[v]
        for e in range(ro[v], ro[v + 1]):
            want += 1
            if lo + w_s[e] >= best:
                break
            if member[col_s[e]]:
                best = min(best, dist[col_s[e]] + w_s[e])
    assert pull_scan_edges(ro, col_s, w_s, dist, member, lo, thr) == (want, cands)
