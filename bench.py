"""Benchmark: direction-optimising BFS (and SSSP) GTEPS on RMAT scale 22.

Workload (one step): a direction-optimising BFS (hybrid heuristic,
alpha=15, beta=24) from each of 64 sources drawn uniformly among the vertices
with degree > 0 (seed 3) on RMAT scale 22, edge factor 16,
(a,b,c,d) = (0.57, 0.19, 0.19, 0.05), symmetrised, self-loops and
duplicates removed, uint32 CSR, seed 1, float32 weights on (0,1] (seed 2).
The graph is synthetic (no dataset) and resident in HBM before timing.

value  = GTEPS = sum over the step's traversals of the edges incident to
         reached vertices / device time (CUDA events), all ranks.
e2e    = the same metric through the C ABI with host buffers: the source ids
         are copied from pinned host memory and every depth array is read back
         to pinned host memory inside the timed region (two instances on two
         streams, each traversal's copy overlapping the next traversal).
roofline: the BFS kernel against the measured HBM copy bandwidth, with
         B = 4(n+1) + 4m + 4n algorithmic bytes per traversal.
cpu_baseline: the oracle's OpenMP frontier BFS on the host cores, a bounded
         sample of the same workload.

Multi-GPU (torchrun): replicas; each rank holds the graph and runs its own 64
sources (weak scaling); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SCALE, EDGE_FACTOR, A, B, C = 22, 16, 0.57, 0.19, 0.19
RMAT_ABC = (A, B, C)  # main() binds the name C to ctypes
GRAPH_SEED, WEIGHT_SEED, SOURCE_SEED = 1, 2, 3
N_SOURCES = 64
ALPHA, BETA = 15.0, 24.0
# batched BFS: pull once the frontier's out-degree exceeds a quarter of the
# in-degree of the vertices some source has not reached (alpha 4: 3.16 ms
# against 4.75 ms at alpha 1 for 64 sources on RMAT-22); push again below n/beta
MS_ALPHA, MS_BETA = 4.0, 24.0
BC_SCALE, BC_SOURCES = 20, 64
METRIC = "BFS/SSSP GTEPS & %HBM roofline on RMAT-22; learned+batched vs plain speedup"


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(name: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(name)
        except Exception:
            return None
    return None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every 20 ms during
    the timed region, through NVML (read-only queries); nvidia-smi when NVML
    is unavailable."""

    # NVML clock-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, index: int):
        self.index = index
        self.rows = []  # (sm_mhz, max_mhz, reason bits)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _sample_nvml(self):
        p = self._nvml
        h = p.nvmlDeviceGetHandleByIndex(self.index)
        mx = p.nvmlDeviceGetMaxClockInfo(h, p.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                sm = p.nvmlDeviceGetClockInfo(h, p.NVML_CLOCK_SM)
                bits = p.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((float(sm), float(mx), int(bits)))
            except Exception:
                pass
            self._stop.wait(0.02)

    def _sample_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.sw_power_cap,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.hw_thermal_slowdown")
        bitv = [0x4, 0x8, 0x20, 0x40]
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                bits = sum(b for b, s in zip(bitv, f[2:]) if s == "Active")
                self.rows.append((float(f[0]), float(f[1]), bits))
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            target = self._sample_nvml
        except Exception:
            target = self._sample_smi
        self._t = threading.Thread(target=target, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        sm = [r[0] for r in self.rows]
        reasons = sorted({name for r in self.rows for b, name in self.REASONS.items() if r[2] & b})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[1] for r in self.rows) if self.rows else None,
                "reasons": reasons, "samples": len(self.rows), "source": "nvml" if self._nvml else "nvidia-smi"}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_graph(sg):
    t = time.time()
    g = sg.io.rmat(SCALE, EDGE_FACTOR, A, B, C, seed=GRAPH_SEED, weight_seed=WEIGHT_SEED, perm_seed=0,
                   value_type=sg.WEIGHT_F32)
    return g, time.time() - t


def bench_config(n: int, m: int) -> dict:
    """The workload as both arms report it (identical keys and values)."""
    return {"workload": f"DO-BFS (hybrid, alpha {ALPHA:g}, beta {BETA:g}) from {N_SOURCES} random sources per GPU, "
                        f"RMAT-{SCALE} ef{EDGE_FACTOR} (0.57,0.19,0.19,0.05) seed 1",
            "n": n, "m": m, "sources_per_step": N_SOURCES, "source_seed": SOURCE_SEED,
            "l2": "inputs larger than L2 (CSR %.2f GB > 126 MB)" % ((4 * (n + 1) + 8 * m) / 1e9)}


def run_reference(args, world, rank):
    """CPU arm: the oracle's OpenMP restatement of BFS::run (the reference is
    SYCL and cannot be compiled here) on all host cores, on the same workload
    as the GPU arm: the same RMAT-22 graph (built by the oracle's copy of the
    generator, so this process loads nothing of sygraph_b200) and the same 64
    sources per step."""
    if rank != 0:
        return
    import oracle
    t0 = time.time()
    g = oracle.rmat(SCALE, EDGE_FACTOR, A, B, C, seed=GRAPH_SEED, weight_seed=WEIGHT_SEED, perm_seed=0, value_type=1)
    gen_s = time.time() - t0
    srcs = oracle.sample_sources(g, N_SOURCES, seed=SOURCE_SEED)
    cores = os.cpu_count() or 1
    reached = {}

    def step():
        edges = 0
        t = time.perf_counter()
        for s in srcs:
            d, _, _ = oracle.bfs_frontier(g, int(s), 2, ALPHA, BETA, nthreads=cores)
            reached[int(s)] = oracle.visited_edges(g, d, g.n + 1)
            edges += reached[int(s)]
        return edges, time.perf_counter() - t

    for _ in range(args.warmup):
        step()
    tot_e, tot_t = 0, 0.0
    for _ in range(args.steps):
        e, dt = step()
        tot_e += e
        tot_t += dt
    val = tot_e / tot_t / 1e9
    line = {"metric": METRIC, "value": val, "unit": "GTEPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_t / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "uint32", "data": "synthetic",
            "impl": "reference", "config": bench_config(g.n, g.m),
            "graph": {"generate_s": round(gen_s, 2), "generator": "oracle.rmat (the product generator restated)"},
            "cpu_baseline": {"value": val, "unit": "GTEPS", "cores": cores, "kind": "port",
                             "sample": f"the whole workload: {N_SOURCES} hybrid BFS traversals per step on "
                                       f"RMAT-{SCALE}, OpenMP oracle with {cores} threads"},
            "e2e": {"value": val, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is SYCL and cannot be compiled here (no SYCL compiler); the oracle's OpenMP "
                    "restatement of its BFS::run (algorithms/bfs.hpp:153-350) is timed instead"}
    print(json.dumps(line), flush=True)


def cc_fixed_point(csr, labels) -> bool:
    """Max-label components on a symmetric graph, checked without a second
    implementation: equal labels across every edge, every label at least the
    vertex id, and every label the id of a vertex that carries it."""
    ro = csr.row_offsets.astype(np.int64)
    src = np.repeat(np.arange(csr.n, dtype=np.int64), np.diff(ro))
    lab = labels.astype(np.int64)
    return bool((lab[src] == lab[csr.column_indices]).all() and (lab >= np.arange(csr.n)).all()
                and (lab[lab] == lab).all())


def dag_wedges(csr) -> tuple[int, int]:
    """Over the degree-ordered DAG's edges (u,v): the sum of min(d+(u), d+(v))
    (the set probes of the triangle count, which streams each edge's shorter
    row) and the sum of d+(v) (head rows only); numpy, outside the timed
    region."""
    ro = csr.row_offsets.astype(np.int64)
    col = csr.column_indices.astype(np.int64)
    deg = np.diff(ro)
    src = np.repeat(np.arange(csr.n, dtype=np.int64), deg)
    keep = (deg[src] < deg[col]) | ((deg[src] == deg[col]) & (src < col))
    dplus = np.bincount(src[keep], minlength=csr.n)
    a, b = dplus[src[keep]], dplus[col[keep]]
    return int(np.minimum(a, b).sum()), int(b.sum())


def _launch_ms(torch, fn) -> float:
    """Device time of what `fn` enqueues, by CUDA events on the current stream."""
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b)


def _alternating_ms(torch, runs, sources, reps: int = 6):
    """Device time per launch of each of `runs` (functions of a source that
    enqueue one launch): each source's median over `reps` rounds, averaged
    over the sources.  The runs' launches of a source go back to back on the
    current stream, each between two CUDA events, in reversed order every
    other round, with one host wait per round: every mode sees the same
    clocks and caches."""
    times = [[[] for _ in sources] for _ in runs]
    for rep in range(reps + 1):  # the first round warms up
        pairs = []
        order = list(enumerate(runs)) if rep % 2 == 0 else list(enumerate(runs))[::-1]
        for i, s in enumerate(sources):
            for k, run in order:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                run(int(s))
                b.record()
                pairs.append((k, i, a, b))
        torch.cuda.synchronize()
        if rep:
            for k, i, a, b in pairs:
                times[k][i].append(a.elapsed_time(b))
    return [float(np.mean([np.median(t) for t in per_src])) for per_src in times]


def _summary(line: dict) -> dict:
    """The sub-benchmarks' headline figures in one short object, printed as
    the line's last key (the full objects above hold the details)."""
    r3 = lambda x: None if x is None else round(float(x), 3)  # noqa: E731
    b, ss, bc, ln = line["batched"], line["sssp"], line["bc_batched"], line["learned"]
    dl = ss["delta_stepping"]
    out = {
        "bfs_gteps": r3(line["value"]), "bfs_frac": r3(line["roofline"]["frac"]), "e2e_gteps": r3(line["e2e"]["value"]),
        "learned_bfs_rmat22": r3(ln.get("rmat_speedup_vs_heuristic")),
        "learned_bfs_grid4096": r3(ln.get("grid4096_speedup_vs_heuristic")),
        "batched_gteps": r3(b["value"]), "batched_frac": r3(b["roofline"]["frac"]),
        "learned_batched_rmat22": r3(b["learned"]["rmat_speedup_vs_heuristic"]),
        "learned_batched_grid4096": r3(b["learned"]["grid4096_speedup_vs_heuristic"]),
        "sssp_bf_gteps": r3(ss["value"]), "sssp_bf_frac": r3(ss["roofline"]["frac"]),
        "sssp_delta_gteps": r3(dl["value"]), "sssp_delta_frac": r3(dl["roofline"]["frac"]),
        "learned_sssp_rmat22": r3(dl["learned"]["speedup_vs_rule"]),
        "bc_batched_ms": r3(bc.get("launch_ms")), "bc_vs_per_source": r3(bc.get("speedup_vs_per_source")),
        "parity_ok": (line.get("parity") or {}).get("ok"),
    }
    sv = line.get("serving")
    if sv:
        r = sv["runs"][0]
        out.update({"serve_qps": r3(r["qps_served"]), "serve_p99_ms": r3(r["p99_ms"]),
                    "serve_bfs_p99_ms": r3(r["bfs"]["p99_ms"]),
                    "serve_vs_one_at_a_time": r3(sv["served_qps_vs_one_at_a_time"])})
    return out


def cpu_baseline(g, srcs):
    """The oracle's OpenMP frontier BFS on the host cores over a bounded
    sample of the bench's sources (about 15 s); returns the baseline object
    and the oracle's depths per source (the bench's parity check)."""
    import oracle
    cores = os.cpu_count() or 1
    edges, t0 = 0, time.perf_counter()
    depths = {}
    for s in srcs:
        d, _, _ = oracle.bfs_frontier(g, int(s), 2, ALPHA, BETA, nthreads=cores)
        edges += oracle.visited_edges(g, d, g.n + 1)
        depths[int(s)] = d
        if time.perf_counter() - t0 > 15.0:
            break
    dt = time.perf_counter() - t0
    return {"value": edges / dt / 1e9, "unit": "GTEPS", "cores": cores, "kind": "port",
            "sample": f"{len(depths)} hybrid BFS traversals (alpha 15, beta 24) on RMAT-{SCALE}, OpenMP oracle"}, depths


PARITY_SOURCES = 8


def bench_parity(sg, g, bfs, srcs, ref_depths, mb_rows, sssp_first) -> dict:
    """The GPU results of this run against the oracle on the bench's own graph
    and sources: the single-source depths and the batched launch's rows for
    every source the CPU baseline traversed, and the first source's SSSP
    distances (delta-stepping, fp32 bits) against Dijkstra."""
    import oracle
    bfs_ok = True
    for s, want in ref_depths.items():
        bfs.init(s)
        bfs.run(2, ALPHA, BETA)
        bfs_ok &= bool(np.array_equal(bfs.getDistances(), want))
    rows_ok = all(bool(np.array_equal(mb_rows[i], ref_depths[int(s)]))
                  for i, s in enumerate(srcs[:len(mb_rows)]) if int(s) in ref_depths)
    dref = oracle.sssp_dijkstra(g, int(srcs[0]))
    sssp_ok = bool(np.array_equal(sssp_first.view(np.uint32), dref.view(np.uint32)))
    return {"ok": bool(bfs_ok and rows_ok and sssp_ok), "bfs_sources": len(ref_depths), "bfs_depths_equal": bfs_ok,
            "batched_rows_equal": rows_ok, "sssp_sources": 1, "sssp_bits_equal": sssp_ok,
            "oracle": "oracle.bfs_frontier (alpha 15, beta 24) and oracle.sssp_dijkstra"}


def profile_case(kind: str) -> None:
    """Two traversals on the bench graph from the first bench source, for ncu
    captures: the second launch is the one to capture (-s 1 -c 1 on the
    traversal kernel)."""
    import sygraph_b200 as sg
    if kind in ("tc", "cc"):  # on the RMAT-20 graph only
        gbc = sg.io.rmat(BC_SCALE, EDGE_FACTOR, *RMAT_ABC, seed=1)
        Gbc = sg.graph.build.fromCSR(gbc)
        a = sg.algorithms.TC(Gbc) if kind == "tc" else sg.algorithms.CC(Gbc)
        for _ in range(2):
            a.run()
        out = {"triangles": a.getNumTriangles()} if kind == "tc" else {"sweeps": a.iterations}
        print(json.dumps({"profile": kind, **out}))
        return
    g, _ = make_graph(sg)
    src = int(sg.io.sample_sources(g, 1, seed=SOURCE_SEED)[0])
    G = sg.graph.build.fromCSR(g)
    if kind == "bfs":
        a = sg.algorithms.BFS(G)
        for _ in range(2):
            a.init(src)
            det = a.run(2, ALPHA, BETA)
        print(json.dumps({"profile": "bfs", "source": src, "iterations": det.iterations,
                          "levels": a.level_records()}))
    elif kind == "msbfs":
        srcs = sg.io.sample_sources(g, N_SOURCES, seed=SOURCE_SEED)
        a = sg.algorithms.MultiBFS(G, N_SOURCES)
        for _ in range(2):
            det = a.run(srcs, 2, MS_ALPHA, MS_BETA)
        print(json.dumps({"profile": "msbfs", "sources": N_SOURCES, **det}))
    elif kind == "bc":
        gbc = sg.io.rmat(BC_SCALE, EDGE_FACTOR, *RMAT_ABC, seed=1)
        Gbc = sg.graph.build.fromCSR(gbc)
        sbc = sg.io.sample_sources(gbc, BC_SOURCES, seed=SOURCE_SEED)
        a = sg.algorithms.BatchedBC(Gbc)
        for _ in range(2):
            det = a.run(sbc)
        print(json.dumps({"profile": "bc", "sources": BC_SOURCES, **det}))
    else:
        # "sssp": delta-stepping at the bucket width the autotuner picks on
        # this graph; "sssp_bf": the reference's frontier Bellman-Ford
        a = sg.algorithms.SSSP(G)
        delta = SSSP_PROFILE_DELTA if kind == "sssp" else 0.0
        a.set_pull(SSSP_PULL)
        a.set_delta(delta)
        for _ in range(2):
            a.init(src)
            it = a.run()
        print(json.dumps({"profile": kind, "source": src, "delta": delta, "iterations": it}))


SERVE_SCALES = (14, 16, 18, 20, 21, 22, 22, 23)
SERVE_QPS = (1000.0, 3000.0, 6000.0)
SERVE_SECONDS = 2.0
SERVE_SLOTS = 4
SSSP_DELTA = 0.1
SSSP_PULL = 0  # pull iterations off: on RMAT they cost more than the pushes they replace
# delta-stepping bucket width of the ncu capture: the autotuner's pick on the
# RMAT-22 bench graph (its candidates are a factor sqrt(2) apart)
SSSP_PROFILE_DELTA = 0.1 * 2 ** -0.5


def _edge_list(g, seed: int = 5):
    """One direction (u < v) of each pair of a symmetric CSR, shuffled."""
    ro, col = g.row_offsets, g.column_indices
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(ro))
    keep = src < col
    order = np.random.default_rng(seed).permutation(int(keep.sum()))
    return src[keep][order], col[keep][order], g.values[keep][order]


def construction_bench(sg, torch, g) -> dict:
    def wall(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, r

    s, d, w = _edge_list(g)
    build = lambda a, b, c: sg.graph.build.fromCOO(g.n, a, b, c, symmetrize=True, dedupe=True,  # noqa: E731
                                                   drop_self_loops=True)
    t_host_arrays = min(wall(lambda: build(s, d, w))[0] for _ in range(3))
    ds, dd, dw = sg.DeviceArray(s), sg.DeviceArray(d), sg.DeviceArray(w)
    t_dev_arrays, G = wall(lambda: build(ds, dd, dw))
    t_dev_arrays = min([t_dev_arrays] + [wall(lambda: build(ds, dd, dw))[0] for _ in range(2)])
    same = bool(np.array_equal(G.csr.row_offsets, g.row_offsets) and np.array_equal(G.csr.column_indices,
                                                                                      g.column_indices))
    del G, ds, dd, dw
    g20 = sg.io.rmat(20, EDGE_FACTOR, *RMAT_ABC, seed=1)
    s2, d2, w2 = _edge_list(g20)
    t_dev20 = min(wall(lambda: sg.graph.build.fromCOO(g20.n, s2, d2, w2, symmetrize=True, dedupe=True,
                                                     drop_self_loops=True))[0] for _ in range(3))
    t_host20 = wall(lambda: sg.graph.build.fromCSR(sg.io.fromCOO(g20.n, s2, d2, w2, symmetrize=True, dedupe=True,
                                                                  drop_self_loops=True)))[0]
    return {"workload": f"RMAT-{SCALE} edge list ({s.size} pairs, shuffled) -> symmetrised CSR (m {g.m})",
            "device_ms_from_host_arrays": t_host_arrays * 1e3, "device_ms_from_device_arrays": t_dev_arrays * 1e3,
            "identical_csr": same,
            "rmat20": {"pairs": int(s2.size), "device_ms_from_host_arrays": t_dev20 * 1e3,
                       "host_ms": t_host20 * 1e3, "speedup": t_host20 / t_dev20}}


def serving_bench(sg, torch) -> dict:
    """Eight resident RMAT graphs (edge factor 16, float32 weights), Poisson
    BFS/SSSP queries (70/30, uniform graph and source) through the serving
    engine; the same query stream one at a time through the single-query
    entry points.  Results stay on the device (no host copy per query)."""
    from sygraph_b200 import serving
    graphs, Gs = [], []
    for i, sc in enumerate(SERVE_SCALES):
        g = sg.io.rmat(sc, EDGE_FACTOR, *RMAT_ABC, seed=31 + i, weight_seed=41 + i, value_type=sg.WEIGHT_F32)
        graphs.append(g)
        Gs.append(sg.graph.build.fromCSR(g))
    sizes = [g.n for g in graphs]
    srv = serving.Server(slots=SERVE_SLOTS, sssp_delta=SSSP_DELTA)
    gids = [srv.add_graph(G) for G in Gs]
    # every workspace built before any query (a workspace built on first use
    # held up the queries queued behind it)
    prep_t0 = time.perf_counter()
    for gi in gids:
        srv.prepare(gi)
    prepare_s = time.perf_counter() - prep_t0
    warm = serving.make_workload(sizes, 200.0, 1.0, 0.7, seed=5)
    serving.run_open_loop(srv, gids, warm)
    serving.warm_up(srv, gids, sizes, SERVE_SLOTS)
    out = {"graphs": [f"RMAT-{s}" for s in SERVE_SCALES], "slots": SERVE_SLOTS, "sssp_delta": SSSP_DELTA,
           "mix": "70% BFS / 30% SSSP", "prepare_s": prepare_s, "runs": []}
    for qps in SERVE_QPS:
        wl = serving.make_workload(sizes, qps, SERVE_SECONDS, 0.7, seed=int(qps))
        r = serving.run_open_loop(srv, gids, wl)
        out["runs"].append({"qps_offered": qps, **r})
    out["stats"] = srv.stats()
    srv.close()
    wl = serving.make_workload(sizes, 1000.0, 1.0, 0.7, seed=9)
    out["one_at_a_time"] = serving.run_one_at_a_time(Gs, wl, sssp_delta=SSSP_DELTA)
    best = max(r["qps_served"] for r in out["runs"])
    out["served_qps_vs_one_at_a_time"] = best / out["one_at_a_time"]["qps_served"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sygraph_b200", choices=["sygraph_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving sub-benchmark")
    ap.add_argument("--sssp-sources", type=int, default=64)
    ap.add_argument("--profile", choices=["bfs", "sssp", "sssp_bf", "msbfs", "bc", "tc", "cc"], default=None,
                    help="profiling case: build the graph, run 2 traversals of one kind and exit (few launches)")
    args = ap.parse_args()
    world, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.profile:
        profile_case(args.profile)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import sygraph_b200 as sg
    sg._lib.call("sg_set_device", local)

    g, gen_s = make_graph(sg)
    from sygraph_b200 import replicas
    srcs_all = sg.io.sample_sources(g, N_SOURCES * world, seed=SOURCE_SEED)
    srcs = replicas.shard(srcs_all, rank, world, per_rank=N_SOURCES)
    G = sg.graph.build.fromCSR(g)
    bfs = sg.algorithms.BFS(G)
    n, m = g.n, g.m
    algo_bytes = 4 * (n + 1) + 4 * m + 4 * n

    # reached-edge totals (GTEPS numerator) from one untimed pass
    reached = {}
    for s in srcs:
        bfs.init(int(s))
        det = bfs.run(2, ALPHA, BETA)
        reached[int(s)] = det.visited_edges
    step_edges = sum(reached.values())

    # one event pair around every launch of the timed region (created
    # beforehand, recorded on the launching stream without any host wait),
    # for the roofline's per-launch duration
    ev_pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps * len(srcs))]
    ev_it = iter(())

    def step():
        for s in srcs:
            bfs.init(int(s))
            pair = next(ev_it, None)
            if pair:
                pair[0].record()
            bfs.run_async(2, ALPHA, BETA)
            if pair:
                pair[1].record()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    launches0 = sg.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        ev_it = iter(ev_pairs)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        barrier()
        ev_it = iter(())
    launches = sg.launch_count() - launches0
    t_ms = replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    ms_per_step = t_ms / args.steps
    value = step_edges * world * args.steps / (t_ms * 1e-3) / 1e9

    # per-launch duration of the BFS kernel: the event pairs of the timed
    # region (the stream never drains between launches, so a pair spans the
    # launch and its kernel, without host time)
    durs = [a.elapsed_time(b) for a, b in ev_pairs]
    kern_ms = float(np.mean(durs))
    peak, peak_kind = peaks()
    achieved = algo_bytes / (kern_ms * 1e-3) / 1e9
    traffic = ncu_traffic("bfs_kernel")

    # end to end through the C ABI: sources from pinned host memory, depths back to pinned host memory
    import ctypes as C
    hp_src = C.c_void_p()
    sg._lib.call("sg_malloc_host_pinned", 4 * len(srcs), C.byref(hp_src))
    dsrc = C.c_void_p()
    sg._lib.call("sg_malloc_device", 4 * len(srcs), C.byref(dsrc))
    np.ctypeslib.as_array(C.cast(hp_src, C.POINTER(C.c_uint32)), shape=(len(srcs),))[:] = srcs
    host_src = np.ctypeslib.as_array(C.cast(hp_src, C.POINTER(C.c_uint32)), shape=(len(srcs),))

    # two instances on two streams: traversal i's depth copy (on its stream,
    # after its kernel) overlaps traversal i+1's kernel on the other stream;
    # each instance's next kernel waits for its previous copy by stream order
    streams, insts, hp_out, d_depth = [], [], [], []
    for _ in range(2):
        st = C.c_void_p()
        sg._lib.call("sg_stream_create", C.byref(st))
        streams.append(st)
        inst = sg.algorithms.BFS(G)
        inst.set_launch(0, st)
        insts.append(inst)
        hp = C.c_void_p()
        sg._lib.call("sg_malloc_host_pinned", 4 * n, C.byref(hp))
        hp_out.append(hp)
        dd = C.POINTER(C.c_uint32)()
        sg._lib.call("sg_bfs_distances_device", inst.handle, C.byref(dd))
        d_depth.append(dd)

    def e2e_step():
        sg._lib.call("sg_memcpy", dsrc, hp_src, 4 * len(srcs), 0, streams[0])
        for i in range(len(srcs)):
            k = i & 1
            sg._lib.call("sg_bfs_init", insts[k].handle, int(host_src[i]))
            sg._lib.call("sg_bfs_run_async", insts[k].handle, 2, ALPHA, BETA)
            sg._lib.call("sg_memcpy_async", hp_out[k], d_depth[k], 4 * n, 1, streams[k])
        for st in streams:
            sg._lib.call("sg_stream_synchronize", st)

    for _ in range(2):
        e2e_step()
    # the copied-back depths are the traversal's (the last source's, on its instance)
    last = np.ctypeslib.as_array(C.cast(hp_out[(len(srcs) - 1) & 1], C.POINTER(C.c_uint32)), shape=(n,))
    insts[(len(srcs) - 1) & 1].init(int(srcs[-1]))
    insts[(len(srcs) - 1) & 1].run(2, ALPHA, BETA)
    assert np.array_equal(last, insts[(len(srcs) - 1) & 1].getDistances())
    barrier()
    e_steps = max(2, args.steps // 2)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(e_steps):
        e2e_step()
    b.record()  # after both streams were synchronised on the host
    barrier()
    e2e_ms = replicas.max_over_ranks(a.elapsed_time(b), device="cuda")
    e2e_val = step_edges * world * e_steps / (e2e_ms * 1e-3) / 1e9
    sg._lib.call("sg_free_host_pinned", hp_src)
    sg._lib.call("sg_free_device", dsrc)
    for hp in hp_out:
        sg._lib.call("sg_free_host_pinned", hp)
    for x in insts:  # back on the graph's stream before the streams go
        x.set_launch(0, None)
    del insts, inst, d_depth
    for st in streams:
        sg._lib.call("sg_stream_destroy", st)

    # learned selector (committed model) on the same sources, and on a held-out
    # 4096 x 4096 grid with 2% long-range pairs, against the reference heuristic
    from sygraph_b200 import selector
    mlp = selector.Mlp.load()
    learned = {"model": "sygraph_b200/models/selector_b200.npz"}
    bl = sg.algorithms.BFS(G)
    bl.set_selector(mlp)
    # both modes on the one instance (same buffers), alternating per source
    rm_h, rm_l = _alternating_ms(torch, [lambda s: (bl.init(s), bl.run_async(2, ALPHA, BETA)),
                                         lambda s: (bl.init(s), bl.run_async(3, ALPHA, BETA))], srcs)
    same_rmat = True
    for s in srcs[:8]:
        bfs.init(int(s))
        bfs.run(2, ALPHA, BETA)
        bl.init(int(s))
        bl.run(3, ALPHA, BETA)
        same_rmat &= bool(np.array_equal(bfs.getDistances(), bl.getDistances()))
    del bl
    learned.update({"rmat_launch_ms": rm_l, "rmat_heuristic_launch_ms": rm_h,
                    "rmat_speedup_vs_heuristic": rm_h / rm_l, "timing": "per-source median over 6 rounds, "
                    "averaged over the sources; both modes on one instance, alternating back to back on one "
                    "stream", "graph_range": mlp.graph_range, "frontier_range": mlp.frontier_range})
    gg = sg.io.grid(4096, long_range_frac=0.02, seed=103)
    Gg = sg.graph.build.fromCSR(gg)
    bg = sg.algorithms.BFS(Gg)
    bg.set_selector(mlp)
    gsrc = sg.io.sample_sources(gg, 4, seed=SOURCE_SEED)
    same = same_rmat
    for s in gsrc:
        bg.init(int(s))
        bg.run(2, ALPHA, BETA)
        d_h = bg.getDistances()
        bg.init(int(s))
        bg.run(3, ALPHA, BETA)
        same &= bool(np.array_equal(d_h, bg.getDistances()))
    g_h, g_l = _alternating_ms(torch, [lambda s: (bg.init(s), bg.run_async(2, ALPHA, BETA)),
                                       lambda s: (bg.init(s), bg.run_async(3, ALPHA, BETA))], gsrc)
    learned.update({"grid4096_heuristic_ms": g_h, "grid4096_learned_ms": g_l,
                    "grid4096_speedup_vs_heuristic": g_h / g_l, "identical_depths": same})
    del bg, Gg, gg

    # the same 64 sources as one bit-parallel batch (one launch); identical
    # depths.  Grid size and direction threshold from the autotuner, timed on
    # these sources before the measurement.
    from sygraph_b200 import autotune
    mbfs = sg.algorithms.MultiBFS(G, len(srcs))
    ms_tuned = autotune.tune_batched_bfs(mbfs, srcs, reps=2, use_cache=False)
    ms_alpha = float(ms_tuned["alpha"])
    for _ in range(2):
        mbfs.run_async(srcs, 2, ms_alpha, MS_BETA)
    torch.cuda.synchronize()
    mb_ms = []
    for _ in range(max(3, args.steps // 2)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        mbfs.run_async(srcs, 2, ms_alpha, MS_BETA)
        b.record()
        b.synchronize()
        mb_ms.append(a.elapsed_time(b))
    mb_det = mbfs.run(srcs, 2, ms_alpha, MS_BETA)
    mb_rows = mbfs.getDistances()[:PARITY_SOURCES].copy()  # checked against the oracle below
    batched_ms = float(np.median(mb_ms))
    batched_gteps = mb_det["reached_edges"] / (batched_ms * 1e-3) / 1e9
    ms_bytes = 4 * (n + 1) + 4 * m + 4 * n * len(srcs)
    # learned + batched: the batched selector against the batched heuristic,
    # both on this instance, alternating; then on the 4096 x 4096 grid
    from sygraph_b200 import train_selector
    bmlp = selector.Mlp.load(train_selector.BATCHED_MODEL_PATH)
    mbfs.set_selector(bmlp)
    mbfs.run(srcs, 3, ms_alpha, MS_BETA)
    b_same = bool(np.array_equal(mbfs.getDistances()[:PARITY_SOURCES], mb_rows))
    bh, bl_ms = _alternating_ms(torch, [lambda _: mbfs.run_async(srcs, 2, ms_alpha, MS_BETA),
                                        lambda _: mbfs.run_async(srcs, 3, ms_alpha, MS_BETA)], [0], reps=8)
    mbfs.set_selector(None)
    del mbfs
    gg = sg.io.grid(4096, long_range_frac=0.02, seed=103)
    Gg = sg.graph.build.fromCSR(gg)
    mg = sg.algorithms.MultiBFS(Gg, 64)
    mg.set_selector(bmlp)
    gsrc64 = sg.io.sample_sources(gg, 64, seed=SOURCE_SEED)
    mg.run(gsrc64, 2, train_selector.BATCH_ALPHA, MS_BETA)
    d_h = mg.getDistances()
    mg.run(gsrc64, 3, train_selector.BATCH_ALPHA, MS_BETA)
    b_same &= bool(np.array_equal(d_h, mg.getDistances()))
    del d_h
    gh, gl = _alternating_ms(torch, [lambda _: mg.run_async(gsrc64, 2, train_selector.BATCH_ALPHA, MS_BETA),
                                     lambda _: mg.run_async(gsrc64, 3, train_selector.BATCH_ALPHA, MS_BETA)],
                             [0], reps=4)
    del mg, Gg, gg
    batched_learned = {"model": "sygraph_b200/models/selector_msbfs_b200.npz", "rmat_heuristic_ms": bh,
                       "rmat_learned_ms": bl_ms, "rmat_speedup_vs_heuristic": bh / bl_ms,
                       "grid4096_heuristic_ms": gh, "grid4096_learned_ms": gl,
                       "grid4096_speedup_vs_heuristic": gh / gl, "identical_depths": b_same,
                       "frontier_range": bmlp.frontier_range}

    # batched Brandes BC: 64 sources per launch on RMAT-20 against the
    # per-source engine on the same sources (float32, both checked equal within 1e-4)
    gbc = sg.io.rmat(BC_SCALE, EDGE_FACTOR, *RMAT_ABC, seed=1)
    Gbc = sg.graph.build.fromCSR(gbc)
    sbc = sg.io.sample_sources(gbc, BC_SOURCES, seed=SOURCE_SEED)
    bcb = sg.algorithms.BatchedBC(Gbc)
    bc_tuned = autotune.tune_batched_bc(bcb, sbc, reps=1, use_cache=False)
    bc_det = bcb.run(sbc)
    bc_ms = float(np.median([_launch_ms(torch, lambda: bcb.run_async(sbc)) for _ in range(3)]))
    x_bc = bcb.getBC()
    bc1 = sg.algorithms.BC(Gbc)
    bc1.init(sbc)
    bc1_ms = float(np.median([_launch_ms(torch, bc1.run) for _ in range(3)]))  # single runs vary up to 1.7x
    y_bc = bc1.getBC().astype(np.float64)
    bc_rel = float(np.max(np.abs(x_bc - y_bc) / np.maximum(1.0, np.abs(y_bc))))
    bc_line = {"value": bc_det["reached_edges"] / (bc_ms * 1e-3) / 1e9, "unit": "GTEPS", "autotuned": bc_tuned,
               "workload": f"Brandes BC, {BC_SOURCES} sources, RMAT-{BC_SCALE} ef{EDGE_FACTOR}",
               "launch_ms": bc_ms, "per_source_ms": bc1_ms, "speedup_vs_per_source": bc1_ms / bc_ms,
               "max_rel_diff_vs_per_source": bc_rel, "forward_levels": bc_det["iterations"]}
    # forward and backward sweeps each read the CSR once; per vertex and
    # source, sigma and delta are written once and read once (4 bytes each)
    bc_bytes = 2 * (4 * (gbc.n + 1) + 4 * gbc.m) + 16 * gbc.n * BC_SOURCES
    bc_line["roofline"] = {"bound": "hbm", "achieved": bc_bytes / (bc_ms * 1e-3) / 1e9, "unit": "GB/s",
                           "frac": bc_bytes / (bc_ms * 1e-3) / 1e9 / peaks()[0],
                           "bytes_per_launch": bc_bytes, "traffic": ncu_traffic("bc_batch_kernel")}
    # CC and TC on the same RMAT-20 graph, through their instances (which own
    # their workspaces): device time of run_async, median of five after one
    # warm-up run
    cc = sg.algorithms.CC(Gbc)
    cc.set_method(cc.PROPAGATION)
    cc.run()
    prop_sweeps = cc.iterations
    prop_ok = cc_fixed_point(gbc, cc.getLabels())
    prop_ms = float(np.median([_launch_ms(torch, cc.run_async) for _ in range(5)]))
    cc.set_method(cc.AUTO)  # union-find on this undirected graph
    cc.run()
    cc_ok = cc_fixed_point(gbc, cc.getLabels())
    cc_ms = float(np.median([_launch_ms(torch, cc.run_async) for _ in range(5)]))
    cc_bytes = 4 * (gbc.n + 1) + 4 * gbc.m + 8 * gbc.n
    cc_line = {"workload": f"connected components (max-id labels), RMAT-{BC_SCALE} ef{EDGE_FACTOR}", "ms": cc_ms,
               "method": "union-find, smaller roots under larger, one pass over the edges",
               "gteps": gbc.m / (cc_ms * 1e-3) / 1e9, "labels_fixed_point": cc_ok,
               "roofline": {"bound": "hbm", "bytes_one_sweep": cc_bytes, "unit": "GB/s",
                            "achieved": cc_bytes / (cc_ms * 1e-3) / 1e9,
                            "frac": cc_bytes / (cc_ms * 1e-3) / 1e9 / peaks()[0]},
               "propagation": {"ms": prop_ms, "sweeps": prop_sweeps, "labels_fixed_point": prop_ok,
                               "note": "the reference's maximum-label propagation, same labels"}}
    tc = sg.algorithms.TC(Gbc)
    tc.run()
    tc_ms = float(np.median([_launch_ms(torch, tc.run_async) for _ in range(5)]))
    tri = tc.getNumTriangles()
    probes, probes_head = dag_wedges(gbc)
    tc_bytes = 4 * (gbc.n + 1) + 4 * gbc.m // 2
    tc_line = {"workload": f"triangle count on the degree-ordered DAG, RMAT-{BC_SCALE} ef{EDGE_FACTOR}",
               "ms": tc_ms, "triangles": tri, "dag_edges": gbc.m // 2, "set_probes": probes,
               "set_probes_head_rows": probes_head,
               "probes_per_s": probes / (tc_ms * 1e-3), "dag_edges_per_s": (gbc.m // 2) / (tc_ms * 1e-3),
               "roofline": {"bound": "hbm", "bytes": tc_bytes, "unit": "GB/s",
                            "achieved": tc_bytes / (tc_ms * 1e-3) / 1e9,
                            "frac": tc_bytes / (tc_ms * 1e-3) / 1e9 / peaks()[0],
                            "traffic": ncu_traffic("tc_hash_kernel")},
               "note": "DAG build (keep bits, scan, compaction, reverse lists) plus the hash-set intersections, "
                       "one run; set_probes = sum over DAG edges (a,b) of min(d+(a), d+(b)), the shorter rows "
                       "streamed from L2 (head rows only: set_probes_head_rows)"}
    del bcb, bc1, cc, tc, Gbc, gbc

    # graph construction on the device: the bench graph's edge list (one
    # direction of each pair, shuffled, with its weights) -> symmetrised,
    # de-duplicated CSR, checked equal to the generator's; the host path
    # (sg_csr_from_edges + upload) timed on the RMAT-20 edge list only
    construction = construction_bench(sg, torch, g)

    # SSSP on a subset of the same sources (reported beside the BFS line)
    sssp = sg.algorithms.SSSP(G)
    ss_edges, ss_ms = 0, 0.0
    sssp_bytes = 4 * (n + 1) + 8 * m + 4 * n
    k_ss = min(args.sssp_sources, len(srcs))
    for s in srcs[:k_ss]:
        sssp.init(int(s))
        sssp.run_async()
    torch.cuda.synchronize()
    for s in srcs[:k_ss]:
        sssp.init(int(s))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        sssp.run_async()
        b.record()
        b.synchronize()
        ss_ms += a.elapsed_time(b)
        ss_edges += reached[int(s)]
    sssp_gteps = ss_edges / (ss_ms * 1e-3) / 1e9
    sssp_kern = ss_ms / k_ss
    sssp_achieved = sssp_bytes / (sssp_kern * 1e-3) / 1e9
    # delta-stepping on the same sources: the same distances (checked), less
    # work; the bucket width from the autotuner (timed on two other sources)
    sssp.set_pull(SSSP_PULL)
    sssp_delta = float(autotune.tune_sssp(sssp, srcs[-2:], autotune.mean_weight(g), reps=3,
                                          use_cache=False)["delta"]) or SSSP_DELTA
    sssp.set_delta(sssp_delta)
    nf_ms, nf_same = 0.0, True
    d_first = None
    for s in srcs[:k_ss]:
        sssp.init(int(s))
        sssp.run_async()
        d_nf = sssp.getDistances()
        if d_first is None:
            d_first = d_nf
        sssp.set_delta(0.0)
        sssp.init(int(s))
        sssp.run()
        nf_same &= bool(np.array_equal(d_nf.view(np.uint32), sssp.getDistances().view(np.uint32)))
        sssp.set_delta(sssp_delta)
        sssp.init(int(s))
        nf_ms += _launch_ms(torch, sssp.run_async)
    nf_kern = nf_ms / k_ss
    # learned heavy phases (the SSSP model) against the heavy_pull rule on the
    # same sources and instance, alternating launch by launch
    from sygraph_b200 import train_selector
    smdl = selector.Mlp.load(train_selector.SSSP_MODEL_PATH)
    sl_t = {False: [[] for _ in range(k_ss)], True: [[] for _ in range(k_ss)]}
    sl_same = True
    for rep in range(5):
        for i, s in enumerate(srcs[:k_ss]):
            for use_model in ((False, True) if rep % 2 == 0 else (True, False)):
                sssp.set_selector(smdl if use_model else None)
                sssp.init(int(s))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                sssp.run_async()
                b.record()
                b.synchronize()
                if rep:
                    sl_t[use_model][i].append(a.elapsed_time(b))
                if rep == 0 and use_model:
                    sl_same &= bool(np.array_equal(sssp.getDistances().view(np.uint32),
                                                   d_first.view(np.uint32))) if i == 0 else True
    sssp.set_selector(None)
    sl_h = float(np.mean([np.median(t) for t in sl_t[False]]))
    sl_l = float(np.mean([np.median(t) for t in sl_t[True]]))
    sssp_learned = {"model": "sygraph_b200/models/selector_sssp_b200.npz", "heavy_range": smdl.heavy_range,
                    "rule_launch_ms": sl_h, "learned_launch_ms": sl_l, "speedup_vs_rule": sl_h / sl_l,
                    "identical_distances": sl_same}

    serve = None if (args.no_serving or world > 1) else serving_bench(sg, torch)

    if rank == 0:
        base, parity = None, None
        if not (args.no_cpu_baseline or world > 1):
            base, ref_depths = cpu_baseline(g, srcs[:PARITY_SOURCES])
            parity = bench_parity(sg, g, bfs, srcs, ref_depths, mb_rows, d_first)
        line = {
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "uint32", "data": "synthetic",
            "config": bench_config(n, m),
            "graph": {"generate_s": round(gen_s, 2), "device_bytes": G.memory_bytes()},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "bfs_kernel", "bytes_per_launch": algo_bytes, "launch_ms": kern_ms},
            "e2e": {"value": e2e_val, "unit": "GTEPS", "h2d_bytes_per_step": 4 * len(srcs),
                    "d2h_bytes_per_step": 4 * n * len(srcs), "ms_per_step": e2e_ms / e_steps,
                    # the depth rows' copy to the host bounds it: the host link's rate
                    "d2h_gbs": 4 * n * len(srcs) / (e2e_ms / e_steps * 1e-3) / 1e9},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": base,
            "parity": parity,
            "batched": {"value": batched_gteps, "unit": "GTEPS", "sources_per_launch": len(srcs),
                        "autotuned": ms_tuned,
                        "launch_ms": batched_ms, "speedup_vs_single_source": batched_gteps / value,
                        "reached_edges": mb_det["reached_edges"], "reached_edges_single": step_edges,
                        "roofline": {"bound": "hbm", "achieved": ms_bytes / (batched_ms * 1e-3) / 1e9,
                                     "peak": peak, "unit": "GB/s",
                                     "frac": ms_bytes / (batched_ms * 1e-3) / 1e9 / peak,
                                     "bytes_per_launch": ms_bytes, "traffic": ncu_traffic("msbfs_kernel")},
                        "learned": batched_learned},
            "learned": learned,
            "bc_batched": bc_line,
            "construction": construction,
            "cc": cc_line,
            "tc": tc_line,
            "serving": serve,
            "sssp": {"value": sssp_gteps, "unit": "GTEPS", "sources": k_ss, "launch_ms": sssp_kern,
                     "schedule": "frontier Bellman-Ford (the reference's)",
                     "delta_stepping": {"delta": sssp_delta, "delta_source": "autotune.tune_sssp",
                                        "launch_ms": nf_kern,
                                  "value": ss_edges / (nf_ms * 1e-3) / 1e9, "unit": "GTEPS",
                                  "speedup": sssp_kern / nf_kern, "identical_distances": nf_same,
                                  "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s",
                                               "achieved": sssp_bytes / (nf_kern * 1e-3) / 1e9,
                                               "frac": sssp_bytes / (nf_kern * 1e-3) / 1e9 / peak,
                                               "bytes_per_launch": sssp_bytes,
                                               "traffic": ncu_traffic("sssp_kernel")},
                                  "learned": sssp_learned},
                     "roofline": {"bound": "hbm", "achieved": sssp_achieved, "peak": peak, "unit": "GB/s",
                                  "frac": sssp_achieved / peak, "bytes_per_launch": sssp_bytes,
                                  "traffic": ncu_traffic("sssp_kernel_bf")}},
        }
        line["summary"] = _summary(line)  # last key: the tail of the line stays readable
        print(json.dumps(line), flush=True)
    del bfs, sssp, G
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
