"""Training pipeline of the learned BFS strategy selector.

BFS levels are unique, so level L visits the same frontier whichever
strategies ran before it: timing every level under each of the six forced
strategies (one traversal per strategy, repeated, median per level) gives the
full per-level cost table of a (graph, source) pair.  One training sample per
level and strategy run: the twelve features the engine logged for that level
(the same device code computes them at inference) and the six measured
log-times; the loss is masked MSE on log-time and the MLP trains on the GPU
(sg_mlp_train).  Evaluation reports, per traversal, the summed level time of
the heuristic's choices, of the MLP's choices and of the per-level best.

    python -m sygraph_b200.train_selector collect --out data.npz
    python -m sygraph_b200.train_selector train --data data.npz --model selector_b200.npz
    python -m sygraph_b200.train_selector evaluate --data held_out.npz --model selector_b200.npz
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import algorithms, build, io
from .selector import IN, OUT, STRATEGIES, MODEL_PATH, Mlp

HYBRID_ALPHA, HYBRID_BETA = 15.0, 24.0
# the engine keeps the heuristic's choice unless the MLP predicts it at least
# this much slower in log-time (chosen on the training tables: most of the
# gain, no training traversal more than about 1% slower than the heuristic)
MARGIN = 0.05
# the engine skips the inference on frontiers below this fraction of n (the
# heuristic's choice stands there), as kLearnedMinFrontier in the engine
MIN_FRONTIER = 1e-3
# device time one inference adds between two levels (features, three layers,
# the block barrier that publishes the choice, and the slower start of the
# level after it), measured from the level timestamps of RMAT-22 traversals:
# the gap before a consulted level grows by about 1.7 us, the next one by
# about 0.5 us; the consulted frontier and graph ranges trade it against the
# model's gains
INFERENCE_US = 2.2
MAX_LEVELS = 4096

# (name, generator, kwargs): RMAT skews and scales, grids with and without
# long-range pairs, uniform random graphs.  The held-out set uses other seeds
# and larger scales than any training graph.
TRAIN_GRAPHS = [
    ("rmat16", "rmat", dict(scale=16, seed=11)),
    ("rmat18", "rmat", dict(scale=18, seed=12)),
    ("rmat20", "rmat", dict(scale=20, seed=13)),
    ("rmat20_ef8", "rmat", dict(scale=20, edge_factor=8, seed=14)),
    ("rmat21_flat", "rmat", dict(scale=21, a=0.45, b=0.22, c=0.22, seed=15)),
    ("rmat21_skew", "rmat", dict(scale=21, a=0.65, b=0.15, c=0.15, seed=16)),
    ("rmat22", "rmat", dict(scale=22, seed=17)),
    ("uniform20", "rmat", dict(scale=20, a=0.25, b=0.25, c=0.25, seed=18)),
    ("grid512", "grid", dict(side=512, long_range_frac=0.0, seed=19)),
    ("grid1024_lr", "grid", dict(side=1024, long_range_frac=0.02, seed=20)),
    ("grid2048_lr", "grid", dict(side=2048, long_range_frac=0.005, seed=21)),
    ("grid2048_lr2", "grid", dict(side=2048, long_range_frac=0.02, seed=22)),
    ("grid3072_lr1", "grid", dict(side=3072, long_range_frac=0.01, seed=23)),
    ("grid1536_lr3", "grid", dict(side=1536, long_range_frac=0.03, seed=24)),
    ("rmat22_b", "rmat", dict(scale=22, seed=25)),
]
EVAL_GRAPHS = [
    ("rmat22_heldout", "rmat", dict(scale=22, seed=101)),
    ("rmat23", "rmat", dict(scale=23, seed=102)),
    ("grid4096_lr", "grid", dict(side=4096, long_range_frac=0.02, seed=103)),
    ("uniform21", "rmat", dict(scale=21, a=0.25, b=0.25, c=0.25, seed=104)),
]


def make_graph(kind: str, kw: dict):
    return io.rmat(**kw) if kind == "rmat" else io.grid(**kw)


def _forced_levels(bfs, source: int, strategy: int, reps: int):
    """Median level times (us) and the logged features of one forced run."""
    bfs.set_schedule([strategy] * MAX_LEVELS)
    times, feats = [], None
    for _ in range(reps):
        bfs.init(source)
        bfs.run(algorithms.bfs_direction.hybrid, HYBRID_ALPHA, HYBRID_BETA)
        times.append(bfs.level_times_us())
        if feats is None:
            feats = bfs.level_features()
    bfs.set_schedule(None)
    return np.median(np.stack(times), 0), feats


def profile_traversal(bfs, source: int, reps: int = 5) -> dict:
    """Per-level cost table t[L, s] and features for one (graph, source)."""
    t, F = [], []
    for s in range(OUT):
        ts, fs = _forced_levels(bfs, source, s, reps)
        t.append(ts)
        F.append(fs)
    levels = min(len(x) for x in t)
    T = np.stack([x[:levels] for x in t], 1)  # levels x 6
    Fe = np.stack([f[:levels] for f in F], 0)  # 6 x levels x 12
    # the heuristic's own schedule (reference hybrid) on the same source
    bfs.init(source)
    bfs.run(algorithms.bfs_direction.hybrid, HYBRID_ALPHA, HYBRID_BETA)
    h = np.array([r["strategy"] for r in bfs.level_records()][:levels], np.int32)
    return {"T": T, "F": Fe, "heuristic": h}


def collect(graphs, sources_per_graph: int = 6, reps: int = 5, log=print) -> dict:
    """Training samples (X, Y, M, group) plus, per traversal, its cost table,
    the heuristic's schedule and the push/warp run's features, concatenated
    over levels with `offsets` marking each traversal."""
    X, Y, M, group, H, TT, F0 = [], [], [], [], [], [], []
    names = []
    gid = 0
    for name, kind, kw in graphs:
        t0 = time.time()
        csr = make_graph(kind, kw)
        G = build.fromCSR(csr)
        bfs = algorithms.BFS(G)
        bfs.log_features(True)
        srcs = [int(np.argmax(csr.degrees()))] + [int(s) for s in io.sample_sources(csr, sources_per_graph - 1,
                                                                                     seed=gid + 7)]
        for src in srcs:
            p = profile_traversal(bfs, src, reps)
            logT = np.log(np.maximum(p["T"], 0.05))
            for s in range(OUT):
                for L in range(p["T"].shape[0]):
                    X.append(p["F"][s, L])
                    Y.append(logT[L])
                    M.append(np.ones(OUT, np.float32))
                    group.append(gid)
            H.append(p["heuristic"])
            TT.append(p["T"])
            F0.append(p["F"][0])
            names.append(f"{name}:{src}")
            gid += 1
        log(f"{name}: n={csr.n} m={csr.m} sources={len(srcs)} {time.time() - t0:.1f}s")
        del bfs, G
    lens = [len(t) for t in TT]
    return {
        "X": np.asarray(X, np.float32), "Y": np.asarray(Y, np.float32), "M": np.asarray(M, np.float32),
        "group": np.asarray(group, np.int32), "names": np.asarray(names),
        "T": np.concatenate(TT).astype(np.float32), "H": np.concatenate(H).astype(np.int32),
        "F0": np.concatenate(F0).astype(np.float32), "offsets": np.concatenate([[0], np.cumsum(lens)]).astype(np.int64),
    }


# The batched (64-source) BFS's selector: push or pull per level (the
# model's outputs 0 and 2), the batched heuristic (alpha 4, beta 24) as the
# fallback; its own model file.  The cost of an inference is negligible
# against a batched level, so it has no graph range.
BATCHED_MODEL_PATH = MODEL_PATH.parent / "selector_msbfs_b200.npz"
BATCH_ALPHA, BATCH_BETA = 4.0, 24.0
BATCH_ALLOWED = (1 << 0) | (1 << 2)
BATCH_SOURCES = 64


def _forced_batch(mb, srcs, direction: int, reps: int):
    """Median level times (us) and logged features of batched runs with every
    level forced to `direction` (0 push, 2 pull)."""
    mb.set_schedule([direction] * MAX_LEVELS)
    times, feats = [], None
    for _ in range(reps):
        mb.run(srcs, algorithms.bfs_direction.hybrid, BATCH_ALPHA, BATCH_BETA)
        times.append(mb.level_times_us())
        if feats is None:
            feats = mb.level_features()
    mb.set_schedule([])
    return np.median(np.stack(times), 0), feats


def collect_batched(graphs, batches_per_graph: int = 3, reps: int = 5, log=print) -> dict:
    """Cost tables of the batched BFS, in the layout of collect(): per batch
    of BATCH_SOURCES sources the level times under forced push and forced
    pull (strategy columns 0 and 2; the other columns repeat the slower of
    the two and are masked out of the loss), the features of both runs as
    samples, and the batched heuristic's schedule."""
    X, Y, M, group, H, TT, F0 = [], [], [], [], [], [], []
    names = []
    gid = 0
    mask = np.array([(BATCH_ALLOWED >> j) & 1 for j in range(OUT)], np.float32)
    for name, kind, kw in graphs:
        t0 = time.time()
        csr = make_graph(kind, kw)
        G = build.fromCSR(csr)
        mb = algorithms.MultiBFS(G, BATCH_SOURCES)
        mb.log_features(True)
        for b in range(batches_per_graph):
            srcs = io.sample_sources(csr, BATCH_SOURCES, seed=1000 + 17 * gid + b)
            tp, fp = _forced_batch(mb, srcs, 0, reps)
            tq, fq = _forced_batch(mb, srcs, 2, reps)
            levels = min(len(tp), len(tq))
            T = np.empty((levels, OUT), np.float32)
            T[:] = np.maximum(tp[:levels], tq[:levels])[:, None]
            T[:, 0], T[:, 2] = tp[:levels], tq[:levels]
            logT = np.log(np.maximum(T, 0.05))
            for Fx in (fp, fq):
                for L in range(levels):
                    X.append(Fx[L])
                    Y.append(logT[L])
                    M.append(mask)
                    group.append(gid)
            mb.run(srcs, algorithms.bfs_direction.hybrid, BATCH_ALPHA, BATCH_BETA)
            H.append(np.array([r["strategy"] for r in mb.level_records()][:levels], np.int32))
            TT.append(T)
            F0.append(fp[:levels])
            names.append(f"{name}:batch{b}")
            gid += 1
        log(f"{name}: n={csr.n} m={csr.m} batches={batches_per_graph} {time.time() - t0:.1f}s")
        del mb, G
    lens = [len(t) for t in TT]
    return {
        "X": np.asarray(X, np.float32), "Y": np.asarray(Y, np.float32), "M": np.asarray(M, np.float32),
        "group": np.asarray(group, np.int32), "names": np.asarray(names),
        "T": np.concatenate(TT).astype(np.float32), "H": np.concatenate(H).astype(np.int32),
        "F0": np.concatenate(F0).astype(np.float32), "offsets": np.concatenate([[0], np.cumsum(lens)]).astype(np.int64),
    }


# Delta-stepping SSSP's selector: push or pull for each bucket's heavy phase
# (outputs 0 and 2), the heavy_pull rule (pull when the bucket's heavy edges
# times SSSP_RATIO exceed m) as the fallback; its own model file.  A bucket's
# state after its heavy phase is the same by push or by pull, so the forced
# all-push and all-pull runs of a source give its per-phase cost table.
SSSP_MODEL_PATH = MODEL_PATH.parent / "selector_sssp_b200.npz"
SSSP_RATIO = 8
SSSP_ALLOWED = BATCH_ALLOWED
ALWAYS_PULL = 0xFFFFFFFF  # heavy_pull ratio that pulls every heavy phase with a heavy edge


def _sssp_phases(sp, source: int, ratio: int, reps: int):
    """Median heavy-phase times (us), the logged features and the directions
    (0 push / 2 pull) of `reps` runs with the heavy_pull ratio `ratio`."""
    sp.set_heavy_pull(ratio)
    times, feats, dirs = [], None, None
    for _ in range(reps):
        sp.init(source)
        sp.run()
        recs = [r for r in sp.level_records() if r["strategy"] in (4, 6)]
        times.append([(r["t_end_ns"] - r["t_start_ns"]) / 1e3 for r in recs])
        dirs = [2 if r["strategy"] == 6 else 0 for r in recs]
        if feats is None:
            feats = sp.level_features()
    L = min(len(t) for t in times)
    sp.set_heavy_pull(SSSP_RATIO)
    return np.median(np.array([t[:L] for t in times]), 0), feats, dirs


def collect_sssp(graphs, sources_per_graph: int = 4, reps: int = 3, log=print) -> dict:
    """Cost tables of delta-stepping's heavy phases, in the layout of
    collect(): per source the phase times under forced push and forced pull
    (strategy columns 0 and 2; the others repeat the slower and are masked
    out of the loss), both runs' features as samples, and the rule's
    directions.  Delta from the autotuner per graph; graphs whose weighted
    rows are not symmetric (no pull) are skipped."""
    from . import autotune
    X, Y, M, group, H, TT, F0 = [], [], [], [], [], [], []
    names = []
    gid = 0
    mask = np.array([(SSSP_ALLOWED >> j) & 1 for j in range(OUT)], np.float32)
    for name, kind, kw in graphs:
        t0 = time.time()
        csr = make_graph(kind, kw)
        G = build.fromCSR(csr)
        if not G.weight_sorted()[2]:
            log(f"{name}: weighted rows not symmetric, skipped")
            continue
        sp = algorithms.SSSP(G)
        srcs = [int(x) for x in io.sample_sources(csr, sources_per_graph, seed=500 + gid)]
        integer = csr.value_type == io.WEIGHT_U32
        delta = float(autotune.tune_sssp(sp, srcs[:1], autotune.mean_weight(csr), integer=integer, reps=1,
                                         use_cache=False)["delta"])
        sp.set_delta(delta)
        sp.log_features(True)
        for src in srcs:
            tp, fp, _ = _sssp_phases(sp, src, 0, reps)
            tq, fq, _ = _sssp_phases(sp, src, ALWAYS_PULL, reps)
            _, _, h = _sssp_phases(sp, src, SSSP_RATIO, 1)
            L = min(len(tp), len(tq), len(h), len(fp), len(fq))
            if not L:
                continue
            T = np.empty((L, OUT), np.float32)
            T[:] = np.maximum(tp[:L], tq[:L])[:, None]
            T[:, 0], T[:, 2] = tp[:L], tq[:L]
            logT = np.log(np.maximum(T, 0.05))
            for Fx in (fp, fq):
                for i in range(L):
                    X.append(Fx[i])
                    Y.append(logT[i])
                    M.append(mask)
                    group.append(gid)
            H.append(np.array(h[:L], np.int32))
            TT.append(T)
            F0.append(fp[:L])
            names.append(f"{name}:{src}")
            gid += 1
        log(f"{name}: n={csr.n} m={csr.m} delta={delta:g} sources={len(srcs)} {time.time() - t0:.1f}s")
        del sp, G
    lens = [len(t) for t in TT]
    return {
        "X": np.asarray(X, np.float32), "Y": np.asarray(Y, np.float32), "M": np.asarray(M, np.float32),
        "group": np.asarray(group, np.int32), "names": np.asarray(names),
        "T": np.concatenate(TT).astype(np.float32), "H": np.concatenate(H).astype(np.int32),
        "F0": np.concatenate(F0).astype(np.float32), "offsets": np.concatenate([[0], np.cumsum(lens)]).astype(np.int64),
    }


def simulate_sssp(params: np.ndarray, forward, F: np.ndarray, heuristic: np.ndarray,
                  margin: float = MARGIN, heavy_range=None) -> np.ndarray:
    """The learned heavy phases' directions as the engine makes them: on the
    phases whose heavy edges (feature 3, a fraction of m) lie in
    `heavy_range` (None: every phase) the MLP (the previous-direction
    feature following the schedule) picks push or pull, the rule's direction
    standing unless the model predicts it `margin` slower in log-time or a
    feature leaves the trusted range; elsewhere the rule decides."""
    lo_h, hi_h = heavy_range if heavy_range is not None else (0.0, np.inf)
    t0 = params.size - 4 * IN
    lo, hi = params[t0 + 2 * IN:t0 + 3 * IN], params[t0 + 3 * IN:t0 + 4 * IN]
    banned = [j for j in range(OUT) if not (SSSP_ALLOWED >> j) & 1]
    out = np.empty(len(F), np.int32)
    prev = 0
    for L in range(len(F)):
        f = np.array(F[L], np.float32)
        f[10] = 1.0 if prev >= 2 else 0.0
        h = int(heuristic[L])
        if not lo_h <= f[3] <= hi_h or np.any(f < lo) or np.any(f > hi):
            out[L] = h
        else:
            y = np.array(forward(f[None, :]), np.float64)[0]
            y[banned] = np.inf
            best = int(np.argmin(y))
            out[L] = h if y[h] - y[best] <= margin else best
        prev = out[L]
    return out


def _asked_sssp(F, heavy_range) -> int:
    lo, hi = heavy_range if heavy_range is not None else (0.0, np.inf)
    return int(np.sum((F[:, 3] >= lo) & (F[:, 3] <= hi))) if len(F) else 0


def heavy_range(mlp, data: dict, cost_us: float = INFERENCE_US):
    """The range of a bucket's heavy edges (fraction of m) on which asking the
    model pays on the training tables (time its choices save against the
    rule's, minus cost_us per inference), over a grid of bounds; (1, 0), an
    empty range, when it pays nowhere."""
    best = None
    for lo in (0.0, 1e-3, 0.01, 0.02, 0.04, 0.06, 0.08, 0.1):
        for hi in (0.125, 0.15, 0.2, 0.25, 0.3, 0.5, 1.0):
            if hi <= lo:
                continue
            net = 0.0
            for _, T, H, F in traversals(data):
                c = simulate_sssp(mlp.params, mlp.forward, F, H, heavy_range=(lo, hi))
                idx = np.arange(len(T))
                net += float((T[idx, H] - T[idx, c]).sum()) - cost_us * _asked_sssp(F, (lo, hi))
            if best is None or net > best[0]:
                best = (net, lo, hi)
    return (best[1], best[2]) if best[0] > 0 else (1.0, 0.0)


def evaluate_sssp(mlp, data: dict, cost_us: float = INFERENCE_US) -> dict:
    """Summed heavy-phase time (us) per source under the rule, under the
    model (plus cost_us per inference, made on the phases inside its heavy
    range) and the per-phase best."""
    rows = []
    hr = getattr(mlp, "heavy_range", None)
    for name, T, H, F in traversals(data):
        c = simulate_sssp(mlp.params, mlp.forward, F, H, heavy_range=hr)
        idx = np.arange(len(T))
        asked = _asked_sssp(F, hr)
        rows.append({"traversal": name, "phases": len(T), "inferences": asked,
                     "heuristic_us": float(T[idx, H].sum()),
                     "learned_us": float(T[idx, c].sum()) + cost_us * asked, "best_us": float(T.min(1).sum()),
                     "learned_schedule": "".join(map(str, c)), "heuristic_schedule": "".join(map(str, H))})
    tot = {k: sum(r[k] for r in rows) for k in ("heuristic_us", "learned_us", "best_us", "inferences")}
    tot["speedup_vs_heuristic"] = tot["heuristic_us"] / max(tot["learned_us"], 1e-9)
    tot["regret_learned"] = tot["learned_us"] / max(tot["best_us"], 1e-9) - 1.0
    tot["regret_heuristic"] = tot["heuristic_us"] / max(tot["best_us"], 1e-9) - 1.0
    return {"total": tot, "traversals": rows}


def traversals(data: dict):
    """(name, T[levels,6], heuristic[levels], features[levels,12]) per traversal."""
    o = data["offsets"]
    for i in range(len(o) - 1):
        a, b = int(o[i]), int(o[i + 1])
        yield str(data["names"][i]), data["T"][a:b], data["H"][a:b], data["F0"][a:b]


def heuristic_choice(f, cur: int, alpha: float = HYBRID_ALPHA, beta: float = HYBRID_BETA) -> int:
    """The reference heuristic (bfs.hpp:325-350) from a level's features and
    the direction `cur` of the level just run: push turns to pull when the
    frontier's degree exceeds the unexplored degree / alpha (features 3 and
    4), pull returns to push below n / beta vertices (feature 1)."""
    if cur < 2:
        return 2 if f[3] > f[4] / alpha else 0
    return 0 if f[1] < 1.0 / beta else 2


def simulate_choices(params: np.ndarray, forward, F: np.ndarray, heuristic: np.ndarray,
                     allowed: int = 0x3F, margin: float = MARGIN, min_frontier: float = MIN_FRONTIER,
                     graph_range=None, max_frontier: float = 1.0, alpha: float = HYBRID_ALPHA,
                     beta: float = HYBRID_BETA) -> np.ndarray:
    """The learned mode's schedule on a traversal, as the engine makes it:
    after each level the heuristic's choice given the direction actually run
    (level 0: the recorded one); the MLP (`forward` maps a feature batch to
    predicted log-times; the current-direction feature follows the schedule)
    is asked only where that choice switches direction, the frontier lies in
    [min_frontier, max_frontier] of the vertices and every feature in the
    trusted range, and overrules the heuristic when it predicts the
    heuristic's choice more than `margin` slower; on a graph whose
    mean-degree feature (9) is outside `graph_range` the heuristic decides
    every level."""
    t0 = params.size - 4 * IN
    lo, hi = params[t0 + 2 * IN:t0 + 3 * IN], params[t0 + 3 * IN:t0 + 4 * IN]
    banned = [j for j in range(OUT) if not (allowed >> j) & 1]
    use_model = graph_range is None or not len(F) or graph_range[0] <= F[0][9] <= graph_range[1]
    out = np.empty(len(F), np.int32)
    prev = 0
    for L in range(len(F)):
        f = np.array(F[L], np.float32)
        if L > 0:
            f[10] = 1.0 if prev >= 2 else 0.0
        h = int(heuristic[0]) if L == 0 else heuristic_choice(F[L], prev, alpha, beta)
        switch = L > 0 and (h >= 2) != (prev >= 2)
        if (not use_model or not switch or f[1] < min_frontier or f[1] > max_frontier or np.any(f < lo)
                or np.any(f > hi)):
            out[L] = h
        else:
            y = np.array(forward(f[None, :]), np.float64)[0]
            y[banned] = np.inf
            best = int(np.argmin(y))
            out[L] = h if np.isfinite(y[h]) and y[h] - y[best] <= margin else best
        prev = out[L]
    return out


def heuristic_along(F, H, c, alpha: float = HYBRID_ALPHA, beta: float = HYBRID_BETA) -> np.ndarray:
    """The heuristic's choice at each level given the schedule `c` run so far."""
    return np.array([int(H[0]) if L == 0 else heuristic_choice(F[L], int(c[L - 1]), alpha, beta)
                     for L in range(len(F))], np.int32)


def consulted(F, c, lo: float, hi: float, alpha: float = HYBRID_ALPHA, beta: float = HYBRID_BETA) -> np.ndarray:
    """Levels at which the engine asks the model along schedule `c`: the
    heuristic switches direction there and the frontier is inside [lo, hi]."""
    h = heuristic_along(F, np.zeros(len(F), np.int32), c, alpha, beta)
    return np.array([L > 0 and (h[L] >= 2) != (c[L - 1] >= 2) and lo <= F[L][1] <= hi
                     for L in range(len(F))], bool)


def evaluate(mlp: Mlp, data: dict, allowed: int = 0x3F, alpha: float = HYBRID_ALPHA,
             beta: float = HYBRID_BETA, cost_us: float = 0.0) -> dict:
    """Summed level time (us) per traversal under the heuristic's schedule,
    the MLP's schedule (plus cost_us per inference it makes) and the
    per-level best; totals and regret."""
    rows = []
    params = mlp.params
    fr = mlp.frontier_range or (MIN_FRONTIER, 1.0)
    g = mlp.graph_range
    for name, T, H, F in traversals(data):
        c = simulate_choices(params, mlp.forward, F, H, allowed, graph_range=g, min_frontier=fr[0],
                             max_frontier=fr[1], alpha=alpha, beta=beta)
        use = g is None or not len(F) or g[0] <= F[0][9] <= g[1]
        asked = int(consulted(F, c, fr[0], fr[1], alpha, beta).sum()) if use else 0
        idx = np.arange(len(T))
        rows.append({"traversal": name, "levels": len(T), "heuristic_us": float(T[idx, H].sum()),
                     "learned_us": float(T[idx, c].sum()) + cost_us * asked, "best_us": float(T.min(1).sum()),
                     "inferences": asked, "learned_schedule": "".join(map(str, c)),
                     "heuristic_schedule": "".join(map(str, H))})
    tot = {k: sum(r[k] for r in rows) for k in ("heuristic_us", "learned_us", "best_us", "inferences")}
    tot["speedup_vs_heuristic"] = tot["heuristic_us"] / max(tot["learned_us"], 1e-9)
    tot["regret_learned"] = tot["learned_us"] / max(tot["best_us"], 1e-9) - 1.0
    tot["regret_heuristic"] = tot["heuristic_us"] / max(tot["best_us"], 1e-9) - 1.0
    return {"total": tot, "traversals": rows}


def _net_gain(params, forward, T, H, F, lo, hi, allowed, alpha, beta, cost_us) -> float:
    """Time the model's schedule saves on one traversal against the
    heuristic's, minus cost_us per inference."""
    c = simulate_choices(params, forward, F, H, allowed, min_frontier=lo, max_frontier=hi, alpha=alpha, beta=beta)
    h = heuristic_along(F, H, c, alpha, beta)
    idx = np.arange(len(T))
    return float((T[idx, h] - T[idx, c]).sum()) - cost_us * int(consulted(F, c, lo, hi, alpha, beta).sum())


def frontier_range(mlp: Mlp, data: dict, cost_us: float = INFERENCE_US, allowed: int = 0x3F,
                   alpha: float = HYBRID_ALPHA, beta: float = HYBRID_BETA):
    """The frontier-size range (fraction of n) on which consulting the model
    pays on the training traversals: over a grid of bounds, the summed time
    its choices save against the heuristic's, minus cost_us per inference
    made; the best range."""
    params = mlp.params
    best = None
    for lo in (0.0, 1e-4, 3e-4, 1e-3, 3e-3, 1e-2, 2e-2, 3e-2, 5e-2):
        for hi in (0.05, 0.1, 0.2, 0.3, 0.5, 1.0):
            if hi <= lo:
                continue
            net = sum(_net_gain(params, mlp.forward, T, H, F, lo, hi, allowed, alpha, beta, cost_us)
                      for _, T, H, F in traversals(data))
            if best is None or net > best[0]:
                best = (net, lo, hi)
    return (best[1], best[2])


def graph_range(mlp: Mlp, data: dict, widen: float = 0.05, cost_us: float = INFERENCE_US, allowed: int = 0x3F,
                alpha: float = HYBRID_ALPHA, beta: float = HYBRID_BETA):
    """The range of the mean-degree feature (9, constant per graph) over the
    training graphs on which consulting the model pays (its schedules save
    more than cost_us per inference, summed over the graph's traversals),
    widened by `widen`: elsewhere the engine never asks it and stages
    nothing.  (1, 0), an empty range, when it pays on no graph."""
    params = mlp.params
    fr = getattr(mlp, "frontier_range", None) or (MIN_FRONTIER, 1.0)
    per_graph = {}
    for name, T, H, F in traversals(data):
        if not len(F):
            continue
        key = name.split(":")[0]
        net = _net_gain(params, mlp.forward, T, H, F, fr[0], fr[1], allowed, alpha, beta, cost_us)
        f9, tot = per_graph.get(key, (float(F[0][9]), 0.0))
        per_graph[key] = (f9, tot + net)
    f9 = [v[0] for v in per_graph.values() if v[1] > 0.0]
    return (min(f9) - widen, max(f9) + widen) if f9 else (1.0, 0.0)


def level_weights(Y: np.ndarray, lo: float = 0.25, hi: float = 8.0) -> np.ndarray:
    """Per-sample loss weights: the square root of the level's best time
    against the median level, clipped to [lo, hi], so that the levels that
    dominate a traversal's time dominate the fit."""
    best = np.exp(Y.min(1))
    return np.clip(np.sqrt(best / np.median(best)), lo, hi).astype(np.float32)


def train(data: dict, steps: int = 6000, lr: float = 3e-3, seed: int = 0, weighted: bool = True) -> Mlp:
    """Fit the MLP on the GPU; normalisation and trusted range from X."""
    X, Y, M = data["X"], data["Y"], data["M"]
    if weighted:
        M = (M * level_weights(Y)[:, None]).astype(np.float32)
    rng = np.random.default_rng(seed)
    I, H, O = IN, 32, OUT
    p = np.zeros(H * I + H + H * H + H + O * H + O + 4 * I, np.float32)
    # He-uniform initialisation of the trainable block
    k = 0
    for rows, cols in ((H, I), (H, H), (O, H)):
        lim = np.sqrt(6.0 / cols)
        p[k:k + rows * cols] = rng.uniform(-lim, lim, rows * cols)
        k += rows * cols + rows
    p[k - O:k] = float(Y.mean())  # output bias starts at the mean log-time
    mlp = Mlp(p)
    mlp.set_normalisation(X)
    mlp.train(X, Y, M, steps=steps, lr=lr)
    return mlp


def _save(data: dict, path: str) -> None:
    np.savez_compressed(path, **data)


def _load(path: str) -> dict:
    with np.load(path) as d:
        return {k: d[k] for k in d.files}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--out", required=True)
    c.add_argument("--set", choices=["train", "eval"], default="train")
    c.add_argument("--batched", action="store_true", help="the 64-source batched BFS (push / pull per level)")
    c.add_argument("--sssp", action="store_true", help="delta-stepping SSSP's heavy phases (push / pull per bucket)")
    c.add_argument("--sources", type=int, default=6)
    c.add_argument("--reps", type=int, default=5)
    t = sub.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--model", default=None)
    t.add_argument("--batched", action="store_true")
    t.add_argument("--sssp", action="store_true")
    t.add_argument("--steps", type=int, default=6000)
    t.add_argument("--lr", type=float, default=3e-3)
    r = sub.add_parser("regate", help="recompute a model's frontier and graph ranges on training tables")
    r.add_argument("--data", required=True)
    r.add_argument("--model", default=None)
    r.add_argument("--batched", action="store_true")
    r.add_argument("--sssp", action="store_true")
    r.add_argument("--cost-us", type=float, default=INFERENCE_US)
    e = sub.add_parser("evaluate")
    e.add_argument("--data", required=True)
    e.add_argument("--model", default=None)
    e.add_argument("--batched", action="store_true")
    e.add_argument("--sssp", action="store_true")
    e.add_argument("--json", default=None)
    e.add_argument("--cost-us", type=float, default=INFERENCE_US)
    a = ap.parse_args(argv)
    if a.cmd == "collect":
        graphs = TRAIN_GRAPHS if a.set == "train" else EVAL_GRAPHS
        if a.sssp:
            _save(collect_sssp(graphs), a.out)
        elif a.batched:
            _save(collect_batched(graphs, reps=a.reps), a.out)
        else:
            _save(collect(graphs, a.sources, a.reps), a.out)
        return 0
    model = a.model or str(SSSP_MODEL_PATH if a.sssp else BATCHED_MODEL_PATH if a.batched else MODEL_PATH)
    kw = dict(allowed=BATCH_ALLOWED, alpha=BATCH_ALPHA, beta=BATCH_BETA) if a.batched else {}
    data = _load(a.data)
    if a.sssp:
        # asked on the buckets inside its heavy range: no frontier or graph range
        mlp = train(data, a.steps, a.lr) if a.cmd == "train" else Mlp.load(model)
        cost = getattr(a, "cost_us", INFERENCE_US)
        if a.cmd in ("train", "regate"):
            mlp.heavy_range = heavy_range(mlp, data, cost)
        rep = evaluate_sssp(mlp, data, cost)
        if a.cmd in ("train", "regate"):
            mlp.save(model, strategies=np.asarray(STRATEGIES), train_report=json.dumps(rep["total"]))
        print(json.dumps(rep["total"]))
        if getattr(a, "json", None):
            with open(a.json, "w") as f:
                json.dump(rep, f, indent=1)
        return 0
    if a.cmd in ("train", "regate"):
        mlp = train(data, a.steps, a.lr) if a.cmd == "train" else Mlp.load(model)
        cost = getattr(a, "cost_us", INFERENCE_US)
        mlp.frontier_range = frontier_range(mlp, data, cost, **kw)
        mlp.graph_range = None if a.batched else graph_range(mlp, data, cost_us=cost, **kw)
        rep = evaluate(mlp, data, cost_us=cost, **kw)
        mlp.save(model, strategies=np.asarray(STRATEGIES), train_report=json.dumps(rep["total"]))
        print(json.dumps({"frontier_range": mlp.frontier_range, "graph_range": mlp.graph_range, **rep["total"]}))
    else:
        rep = evaluate(Mlp.load(model), data, cost_us=a.cost_us, **kw)
        print(json.dumps(rep["total"]))
        if a.json:
            with open(a.json, "w") as f:
                json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
