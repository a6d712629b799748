"""A synchronous CPU model of the near-far (delta-stepping) schedule that
sssp_kernel runs: light push steps inside a bucket until its frontier is
empty, one heavy phase over the bucket's members, then a refill of the far
vertices below the next threshold (jumping to the far set's minimum when
none is).  It counts the work per bucket -- light steps, light-edge
relaxations, the members' distinct light edges, heavy edges -- so a schedule
can be judged by its work before it is built.  Each step relaxes against the
distances at its start (the kernel's steps see each other's updates within a
step, so its frontiers can be slightly smaller); the distances are the
least fixed point either way and equal the oracle's Dijkstra.

Usage: ``python tests/bucket_model.py SCALE DELTA [SOURCE]`` prints one line
per bucket on the bench's RMAT graph (seed 1, float weights from seed 2).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np


def _edges(ro, deg, F, keep_w, w):
    d = deg[F]
    tot = int(d.sum())
    if tot == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    starts = np.repeat(ro[F], d)
    e = starts + (np.arange(tot) - np.repeat(np.cumsum(d) - d, d))
    sv = np.repeat(F, d)
    keep = keep_w(w[e])
    return sv[keep], e[keep]


def near_far_model(csr, src: int, delta: float):
    """Returns (distances as float32 with n+1 for unreached, per-bucket work
    as a list of dicts)."""
    ro = np.asarray(csr.row_offsets, np.int64)
    col = np.asarray(csr.column_indices, np.int64)
    w = np.asarray(csr.values, np.float32)
    n = len(ro) - 1
    deg = np.diff(ro)
    dist = np.full(n, np.inf, np.float32)
    dist[src] = 0
    far = np.zeros(n, bool)
    thr = np.float32(delta)
    F = np.array([src], np.int64)
    buckets = []
    while True:
        b = {"threshold": float(thr), "light_steps": 0, "light_relaxations": 0}
        members = []
        while len(F):
            members.append(F)
            sv, e = _edges(ro, deg, F, lambda x: x < delta, w)
            b["light_steps"] += 1
            b["light_relaxations"] += int(len(e))
            u = col[e]
            nd = dist[sv] + w[e]
            c = nd < dist[u]
            if c.any():
                np.minimum.at(dist, u[c], nd[c])
            t = np.unique(u[c])
            near = t[dist[t] < thr]
            far[t[dist[t] >= thr]] = True
            far[near] = False
            F = near
        M = np.unique(np.concatenate(members))
        b["members"] = int(len(M))
        b["member_light_edges"] = int(len(_edges(ro, deg, M, lambda x: x < delta, w)[1]))
        sv, e = _edges(ro, deg, M, lambda x: x >= delta, w)
        b["heavy_edges"] = int(len(e))
        u = col[e]
        nd = dist[sv] + w[e]
        c = nd < dist[u]
        if c.any():
            np.minimum.at(dist, u[c], nd[c])
        far[u[c]] = True
        buckets.append(b)
        while True:
            fv = np.nonzero(far)[0]
            nxt = np.float32(thr + np.float32(delta))
            near = fv[dist[fv] < nxt]
            thr = nxt
            if len(near) or not len(fv):
                break
            thr = max(thr, dist[fv].min())
        if not len(near):
            break
        far[near] = False
        F = near
    return np.where(np.isinf(dist), np.float32(n + 1), dist).astype(np.float32), buckets


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import oracle

    scale, delta = int(sys.argv[1]), float(sys.argv[2])
    g = oracle.rmat(scale, 16, seed=1, weight_seed=2, perm_seed=0, value_type=1)
    src = int(sys.argv[3]) if len(sys.argv) > 3 else int(oracle.sample_sources(g, 1, seed=3)[0])
    d, bk = near_far_model(g, src, delta)
    exact = bool(np.array_equal(d.view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32)))
    print(json.dumps({"scale": scale, "delta": delta, "source": src, "m": int(g.m), "equal_to_dijkstra": exact,
                      "buckets": len(bk), "light_steps": sum(b["light_steps"] for b in bk)}))
    for i, b in enumerate(bk):
        print(json.dumps({"bucket": i, **b}))
