"""Query serving with continuous batching: the Python face of sg_server.

    srv = Server(slots=4, sssp_delta=0.3)
    gid = srv.add_graph(G)
    t = srv.submit(gid, "bfs", source, out)      # out: pinned host buffer or None
    res = srv.wait(t)                            # status, batch size, latency
    srv.stats()

`run_open_loop` drives a server with Poisson arrivals (a fixed-rate open
loop, the arrival times drawn before the run) and reports throughput and
latency percentiles; `run_one_at_a_time` runs the same queries through the
single-query entry points, one after another, for comparison.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call, lib
from .core import WEIGHT_F32, Graph

KINDS = {"bfs": 0, "sssp": 1}


class PinnedBuffer:
    """Page-locked host memory (sg_malloc_host_pinned) viewed as a numpy array."""

    def __init__(self, n: int, dtype):
        self.dtype = np.dtype(dtype)
        self.nbytes = max(1, int(n) * self.dtype.itemsize)
        p = C.c_void_p()
        call("sg_malloc_host_pinned", self.nbytes, C.byref(p))
        self.ptr = p
        self.array = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(self.nbytes,)).view(self.dtype)[:n]

    def __del__(self):
        if getattr(self, "ptr", None) and lib is not None:
            lib.sg_free_host_pinned(self.ptr)
            self.ptr = None


class Server:
    def __init__(self, slots: int = 4, max_batch: int = 64, min_batch: int = 16, ctas_per_slot: int = 0,
                 memory_budget: int = 0, sssp_delta: float = 0.0):
        cfg = _lib.ServerConfig(slots, max_batch, min_batch, ctas_per_slot, memory_budget, sssp_delta)
        h = C.c_void_p()
        call("sg_server_create", C.byref(cfg), C.byref(h))
        self.handle = h
        self.graphs: list[Graph] = []

    def add_graph(self, G: Graph) -> int:
        gid = C.c_uint32()
        call("sg_server_add_graph", self.handle, G.handle, C.byref(gid))
        self.graphs.append(G)
        return gid.value

    def prepare(self, graph_id: int) -> None:
        """Creates every workspace the graph's queries can use on every slot
        now (within the memory budget, without evicting), so that no query
        waits for one to be built."""
        call("sg_server_prepare", self.handle, graph_id)

    def submit(self, graph_id: int, kind: str, source: int, out=None) -> int:
        t = C.c_uint64()
        ptr = None if out is None else C.c_void_p(out.ptr.value if isinstance(out, PinnedBuffer) else out.ctypes.data)
        call("sg_server_submit", self.handle, graph_id, KINDS[kind], int(source), ptr, C.byref(t))
        return t.value

    def wait(self, ticket: int, timeout_s: float = 60.0) -> dict:
        r = _lib.QueryResult()
        call("sg_server_wait", self.handle, ticket, timeout_s, C.byref(r))
        d = {k: getattr(r, k) for k, _ in _lib.QueryResult._fields_}
        d["latency_ms"] = (r.end_ns - r.submit_ns) / 1e6
        d["queue_ms"] = (r.start_ns - r.submit_ns) / 1e6
        return d

    def drain(self, timeout_s: float = 120.0) -> None:
        call("sg_server_drain", self.handle, timeout_s)

    def stats(self) -> dict:
        s = _lib.ServerStats()
        call("sg_server_get_stats", self.handle, C.byref(s))
        return {k: int(getattr(s, k)) for k, _ in _lib.ServerStats._fields_}

    def close(self) -> None:
        h = getattr(self, "handle", None)
        if h and lib is not None:
            lib.sg_server_destroy(h)
            self.handle = None

    def __del__(self):
        self.close()


@dataclass
class Workload:
    """A seeded query stream: (arrival offset s, graph index, kind, source)."""
    arrivals: np.ndarray
    graph: np.ndarray
    kind: list
    source: np.ndarray


def make_workload(graph_sizes, qps: float, duration_s: float, bfs_fraction: float = 0.7, seed: int = 1) -> Workload:
    """Poisson arrivals at `qps` for `duration_s`; uniform graph choice and
    uniform sources; BFS with probability `bfs_fraction`, else SSSP."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / qps, size=int(qps * duration_s * 1.5) + 16)
    t = np.cumsum(gaps)
    t = t[t < duration_s]
    g = rng.integers(0, len(graph_sizes), size=t.size)
    kind = ["bfs" if x < bfs_fraction else "sssp" for x in rng.random(t.size)]
    src = np.array([rng.integers(0, graph_sizes[i]) for i in g], np.uint32)
    return Workload(t, g, kind, src)


def percentiles(lat_ms) -> dict:
    a = np.asarray(lat_ms, np.float64)
    if a.size == 0:
        return {"p50_ms": None, "p99_ms": None, "mean_ms": None}
    return {"p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)), "mean_ms": float(a.mean())}


def warm_up(srv: Server, gids, graph_sizes, slots: int, batch: int = 64, seed: int = 0) -> None:
    """Creates every workspace a run may need before it is timed: for each
    graph, `slots` x `batch` BFS queries at once (a batched launch lands on
    every slot) and `slots` SSSP queries, then waits for all of them."""
    rng = np.random.default_rng(seed)
    for gi, n in zip(gids, graph_sizes):
        tickets = [srv.submit(gi, "bfs", int(rng.integers(0, n))) for _ in range(slots * batch)]
        tickets += [srv.submit(gi, "sssp", int(rng.integers(0, n))) for _ in range(slots)]
        for t in tickets:
            srv.wait(t)


def run_open_loop(srv: Server, gids, wl: Workload, outs=None) -> dict:
    """Submits each query at its arrival time (busy-waiting the host clock),
    waits for all, returns throughput and latency percentiles."""
    tickets = []
    t0 = time.perf_counter()
    for i in range(wl.arrivals.size):
        while time.perf_counter() - t0 < wl.arrivals[i]:
            pass
        out = outs[i] if outs is not None else None
        tickets.append(srv.submit(gids[wl.graph[i]], wl.kind[i], int(wl.source[i]), out))
    res = [srv.wait(t) for t in tickets]
    wall = time.perf_counter() - t0
    ok = [r for r in res if r["status"] == 0]
    out = {"queries": len(res), "failed": len(res) - len(ok), "wall_s": wall,
           "qps_offered": wl.arrivals.size / max(wl.arrivals[-1], 1e-9) if wl.arrivals.size else 0.0,
           "qps_served": len(ok) / wall, "mean_batch": float(np.mean([r["batch_size"] for r in ok])) if ok else 0.0}
    out.update(percentiles([r["latency_ms"] for r in ok]))
    out["bfs"] = percentiles([r["latency_ms"] for r in ok if r["kind"] == 0])
    out["sssp"] = percentiles([r["latency_ms"] for r in ok if r["kind"] == 1])
    return out


def run_one_at_a_time(graphs, wl: Workload, sssp_delta: float = 0.0) -> dict:
    """The same queries through BFS / SSSP instances, one after another on
    the default stream (each waits for the previous): service time per query
    and the throughput that gives.  Every instance the stream needs is
    created, and has run one query (which builds its graph's weight-sorted
    adjacency for delta-stepping), before the clock starts, as the server's
    workspaces are before its timed runs."""
    from . import algorithms
    inst = {}
    for i in range(wl.arrivals.size):
        gi, kind = int(wl.graph[i]), wl.kind[i]
        key = (gi, kind)
        if key in inst:
            continue
        if kind == "bfs":
            inst[key] = algorithms.BFS(graphs[gi])
            inst[key].init(0)
            inst[key].run(2, 15.0, 24.0)
        else:
            inst[key] = algorithms.SSSP(graphs[gi])
            inst[key].set_delta(sssp_delta)
            inst[key].init(0)
            inst[key].run()
    times = []
    t0 = time.perf_counter()
    for i in range(wl.arrivals.size):
        gi, kind, s = int(wl.graph[i]), wl.kind[i], int(wl.source[i])
        a = inst[(gi, kind)]
        t = time.perf_counter()
        a.init(s)
        if kind == "bfs":
            a.run(2, 15.0, 24.0)
        else:
            a.run()
        times.append((time.perf_counter() - t) * 1e3)
    wall = time.perf_counter() - t0
    out = {"queries": len(times), "wall_s": wall, "qps_served": len(times) / wall}
    out.update(percentiles(times))
    return out
