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

Usage: ``python tests/bucket_model.py SCALE DELTA [SOURCE] [--pull]`` prints
one line per bucket on the bench's RMAT graph (seed 1, float weights from
seed 2); ``--pull`` adds the edges a pull of each heavy phase would read.
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


def weight_sorted(ro, col, w):
    """Each row's edges by (weight, column), as the kernel's weight-sorted
    rows."""
    n = len(ro) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ro))
    order = np.lexsort((col, w, rows))
    return col[order], w[order]


def pull_scan_edges(ro, col_s, w_s, dist, member, lo, thr):
    """Edges the heavy-phase pull reads: every vertex beyond the threshold
    scans its weight-sorted row from the lightest edge and stops at the
    first weight with lo + w >= best, best being its own distance lowered by
    the members found so far (d[c] + w).  Returns (edges, candidates)."""
    cand = np.nonzero(dist > thr)[0]
    pos = ro[cand].copy()
    end = ro[cand + 1]
    best = dist[cand].astype(np.float32)
    idx = np.nonzero(pos < end)[0]
    scanned = 0
    lo = np.float32(lo)
    while len(idx):
        e = pos[idx]
        we = w_s[e]
        stop = (lo + we) >= best[idx]
        scanned += len(idx)
        c = col_s[e]
        hit = ~stop & member[c]
        if hit.any():
            h = idx[hit]
            best[h] = np.minimum(best[h], dist[c[hit]] + we[hit])
        pos[idx] += 1
        idx = idx[~stop & (pos[idx] < end[idx])]
    return int(scanned), int(len(cand))


def near_far_model(csr, src: int, delta: float, pull_scan: bool = False):
    """Returns (distances as float32 with n+1 for unreached, per-bucket work
    as a list of dicts).  With pull_scan, each bucket also gets the edges a
    pull of its heavy phase would read (heavy_pull_edges, over
    pull_candidates vertices)."""
    ro = np.asarray(csr.row_offsets, np.int64)
    col = np.asarray(csr.column_indices, np.int64)
    w = np.asarray(csr.values, np.float32)
    n = len(ro) - 1
    deg = np.diff(ro)
    if pull_scan:
        col_s, w_s = weight_sorted(ro, col, w)
    dist = np.full(n, np.inf, np.float32)
    dist[src] = 0
    far = np.zeros(n, bool)
    lo, thr = np.float32(0), np.float32(delta)  # the bucket is [lo, thr)
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
        if pull_scan:
            member = np.zeros(n, bool)
            member[M] = True
            b["heavy_pull_edges"], b["pull_candidates"] = pull_scan_edges(ro, col_s, w_s, dist, member, lo, thr)
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
            lo, thr = thr, nxt
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
    args = [a for a in sys.argv[3:] if not a.startswith("--")]
    src = int(args[0]) if args else int(oracle.sample_sources(g, 1, seed=3)[0])
    d, bk = near_far_model(g, src, delta, pull_scan="--pull" in sys.argv)
    exact = bool(np.array_equal(d.view(np.uint32), oracle.sssp_dijkstra(g, src).view(np.uint32)))
    print(json.dumps({"scale": scale, "delta": delta, "source": src, "m": int(g.m), "equal_to_dijkstra": exact,
                      "buckets": len(bk), "light_steps": sum(b["light_steps"] for b in bk)}))
    for i, b in enumerate(bk):
        print(json.dumps({"bucket": i, **b}))
