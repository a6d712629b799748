"""Command-line front end mirroring the reference's example programs
(examples/{bfs,sssp,cc,bc,tc}/*.cpp with examples/include/utils.hpp:41-97):

    python -m sygraph_b200.cli bfs [-b | -m] [-u] [-s SOURCE] [-c] [-p] [-v | -V]
                                   [--advance push|pull|hybrid] [--alpha A] [--beta B] GRAPH
    python -m sygraph_b200.cli {sssp,cc,bc,tc} [same common flags] GRAPH

-b reads the binary CSR ("SYGRCSR" or the legacy headerless layout), -m a
Matrix Market file, otherwise the text COO format of io::coo::fromCOO
(read_coo.hpp:34-80: '%' comments, a "rows cols edges" line, then "u v [w]"
lines; -u adds (v, u) after every (u, v)), turned into a CSR the way
io::csr::fromCOO does (read_csr.hpp:261-300: rows in edge order, no sorting
or de-duplication, n = largest id + 1).  -c checks the result against a CPU
computation of the same definition (BFS levels, Dijkstra in float32 as
examples/sssp/sssp.cpp:23-66, CC's maximum reaching id, Brandes BC in
float64, triangle count), -p prints the result, -v / -V print the timing
summary the reference's profiler prints (kernel time, total GPU time, edge
throughput in MTEPS, utils/profiler.hpp:47-68); -s picks the source (a random
vertex otherwise).  The CPU checks verify the GPU result; they never replace
it."""
from __future__ import annotations

import argparse
import ctypes as C
import heapq
import random
import sys
import time

import numpy as np

from . import _lib
from .core import CSR, WEIGHT_F32, WEIGHT_U32, Properties

_NP = {WEIGHT_F32: np.float32, WEIGHT_U32: np.uint32}


# ------------------------------------------------------------------ reading --
def read_coo_text(path: str, undirected: bool = False, value_type: int = WEIGHT_F32) -> CSR:
    """io::coo::fromCOO then io::csr::fromCOO: rows keep the file's edge order."""
    us, vs, ws = [], [], []
    weighted = False
    with open(path) as f:
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        if not line:
            raise ValueError("could not read the first line of the file")
        for line in f:
            parts = line.split()
            if len(parts) < 2:
                continue
            us.append(int(parts[0]))
            vs.append(int(parts[1]))
            if len(parts) > 2:
                weighted = True
                ws.append(float(parts[2]) if value_type == WEIGHT_F32 else _leading_uint(parts[2]))
            else:
                ws.append(1)
    u = np.asarray(us, np.int64)
    v = np.asarray(vs, np.int64)
    w = np.asarray(ws, _NP[value_type])
    if undirected:  # (u, v) then (v, u), interleaved as read_coo.hpp:66-71
        u, v, w = (np.stack([u, v], 1).ravel(), np.stack([v, u], 1).ravel(), np.repeat(w, 2))
    n = int(max(u.max(initial=-1), v.max(initial=-1)) + 1) if u.size else 0
    order = np.argsort(u, kind="stable")
    ro = np.zeros(n + 1, np.uint32)
    np.cumsum(np.bincount(u, minlength=n), out=ro[1:])
    props = Properties(directed=not undirected, weighted=weighted)
    return CSR(ro, v[order].astype(np.uint32), w[order] if weighted else None, value_type if weighted else None,
               props)


def _leading_uint(text: str) -> int:
    """What an unsigned stream extraction reads from `text`: its leading
    digits ("0.8" -> 0, "12.5" -> 12)."""
    k = 0
    while k < len(text) and text[k].isdigit():
        k += 1
    return int(text[:k]) if k else 0


def read_graph(args, value_type: int) -> CSR:
    from . import io
    if args.binary:
        return io.fromBinary(args.graph, value_type)
    if args.matrix_market:
        return io.fromMM(args.graph, value_type)
    return read_coo_text(args.graph, args.undirected, value_type)


# --------------------------------------------------------------- CPU checks --
def cpu_bfs(csr: CSR, source: int) -> np.ndarray:
    n = csr.n
    ro, col = csr.row_offsets.astype(np.int64), csr.column_indices
    depth = np.full(n, n + 1, np.uint32)
    depth[source] = 0
    frontier = np.array([source], np.int64)
    level = 0
    while frontier.size:
        starts, ends = ro[frontier], ro[frontier + 1]
        lens = ends - starts
        idx = np.repeat(starts - np.cumsum(lens) + lens, lens) + np.arange(lens.sum())
        nb = np.unique(col[idx])
        nb = nb[depth[nb] == n + 1]
        level += 1
        depth[nb] = level
        frontier = nb.astype(np.int64)
    return depth


def cpu_sssp(csr: CSR, source: int) -> np.ndarray:
    """Dijkstra with float32 (or uint32) sums, as the reference's validator."""
    n = csr.n
    t = np.float32 if csr.value_type == WEIGHT_F32 else np.uint32
    ro, col = csr.row_offsets, csr.column_indices
    w = csr.values if csr.values is not None else np.ones(csr.m, t)
    dist = np.full(n, t(n + 1), t)
    dist[source] = t(0)
    pq = [(t(0), source)]
    while pq:
        d, u = heapq.heappop(pq)
        if d > dist[u]:
            continue
        for e in range(int(ro[u]), int(ro[u + 1])):
            v = int(col[e])
            nd = t(d + w[e])
            if nd < dist[v]:
                dist[v] = nd
                heapq.heappush(pq, (nd, v))
    return dist


def cpu_cc(csr: CSR) -> np.ndarray:
    """labels[v] = the largest id among the vertices that reach v."""
    n = csr.n
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(csr.row_offsets))
    lab = np.arange(n, dtype=np.uint32)
    while True:
        new = lab.copy()
        np.maximum.at(new, csr.column_indices, lab[src])
        if np.array_equal(new, lab):
            return lab
        lab = new


def cpu_bc(csr: CSR, sources) -> np.ndarray:
    """Brandes over the given sources, float64 (unweighted shortest paths)."""
    n = csr.n
    ro, col = csr.row_offsets.astype(np.int64), csr.column_indices.astype(np.int64)
    bc = np.zeros(n)
    for s in sources:
        depth = np.full(n, -1, np.int64)
        sigma = np.zeros(n)
        depth[s], sigma[s] = 0, 1.0
        levels = [np.array([s])]
        while True:
            f = levels[-1]
            lens = ro[f + 1] - ro[f]
            idx = np.repeat(ro[f] - np.cumsum(lens) + lens, lens) + np.arange(lens.sum())
            u = np.repeat(f, lens)
            v = col[idx]
            new = v[depth[v] == -1]
            depth[np.unique(new)] = len(levels)
            on = depth[v] == len(levels)
            np.add.at(sigma, v[on], sigma[u[on]])
            nxt = np.unique(v[on])
            if not nxt.size:
                break
            levels.append(nxt)
        delta = np.zeros(n)
        for L in range(len(levels) - 1, 0, -1):
            f = levels[L - 1]
            lens = ro[f + 1] - ro[f]
            idx = np.repeat(ro[f] - np.cumsum(lens) + lens, lens) + np.arange(lens.sum())
            u = np.repeat(f, lens)
            v = col[idx]
            on = depth[v] == L
            np.add.at(delta, u[on], sigma[u[on]] / sigma[v[on]] * (1.0 + delta[v[on]]))
        delta[s] = 0.0
        bc += delta
    return bc


def cpu_tc(csr: CSR) -> int:
    """Triangles of the undirected simple graph the CSR holds."""
    from scipy import sparse
    n = csr.n
    src = np.repeat(np.arange(n), np.diff(csr.row_offsets))
    col = csr.column_indices.astype(np.int64)
    keep = src != col
    a = sparse.coo_matrix((np.ones(int(keep.sum())), (src[keep], col[keep])), shape=(n, n)).tocsr()
    a = ((a + a.T) > 0).astype(np.float64)
    return int(round((a @ a).multiply(a).sum() / 6))


# ---------------------------------------------------------------- commands --
class _Timer:
    """CUDA events on the legacy default stream around a launch."""

    def __init__(self):
        self.start = C.c_void_p()
        self.end = C.c_void_p()

    def __enter__(self):
        _lib.call("sg_event_record", None, C.byref(self.start))
        return self

    def __exit__(self, *exc):
        _lib.call("sg_event_record", None, C.byref(self.end))
        ms = C.c_float()
        _lib.call("sg_event_elapsed_ms", self.start, self.end, C.byref(ms))
        self.ms = float(ms.value)
        _lib.call("sg_event_destroy", self.start)
        _lib.call("sg_event_destroy", self.end)


def _graph_info(G) -> None:
    e = sys.stderr
    n, m = G.getVertexCount(), G.getEdgeCount()
    print("-----------------------------------", file=e)
    print(f"{'Vertex count:':<17}{n:<10}", file=e)
    print(f"{'Edge count:':<17}{m:<10}", file=e)
    print(f"{'Average degree:':<17}{(m // n if n else 0):<10}", file=e)
    print(f"{'Directed:':<17}{('yes' if G.properties.directed else 'no'):<10}", file=e)
    print("-----------------------------------", file=e)


def _device_info() -> None:
    sm, free, total = C.c_int(), C.c_uint64(), C.c_uint64()
    _lib.call("sg_device_info", C.byref(sm), C.byref(free), C.byref(total))
    print(f"[*] Running on: [CUDA] {sm.value} SMs, {total.value / 2**30:.0f} GiB", file=sys.stderr)


def _status(ok: bool) -> str:
    if not sys.stdout.isatty():
        return "Success" if ok else "Failed"
    return "\033[1;32mSuccess\033[0m" if ok else "\033[1;31mFailed\033[0m"


def _validate(fn) -> None:
    t0 = time.perf_counter()
    ok = bool(fn())
    print(f"Validation: [{_status(ok)}] | Validation Time: {int((time.perf_counter() - t0) * 1e3)} ms")


def _profile(args, kernel: str, ms: float, edges: int, steps=None) -> None:
    """The reference profiler's summary (utils/profiler.hpp:47-68); -V lists
    the engine's steps (its per-level or per-phase device timestamps)."""
    if not (args.v or args.V):
        return
    line = f" Kernel [{kernel} x 1] "
    if args.V and steps:
        line += "".join(f"({i}) {t:.4f} ms " for i, t in enumerate(steps)) + "| "
    print(line + f"Time: {ms} ms")
    print(f"Total GPU Time: {ms} ms")
    mteps = edges / 1e6 / (ms / 1e3) if ms > 0 else 0.0
    # the reference's label, kept for scripts that parse it
    print(f"Total Edge-Througput (MTEPS): {mteps} MTEPS")


def _steps_ms(records) -> list:
    return [(r["t_end_ns"] - r["t_start_ns"]) / 1e6 for r in records]


def _source(args, n: int) -> int:
    return args.source if args.source is not None else random.randrange(n)


def run_bfs(args) -> int:
    from . import algorithms
    csr = _read(args, WEIGHT_F32)
    G = _build(csr)
    b = algorithms.BFS(G)
    src = _source(args, csr.n)
    b.init(src)
    mode = {"push": algorithms.bfs_direction.push, "pull": algorithms.bfs_direction.pull,
            "hybrid": algorithms.bfs_direction.hybrid}[args.advance]
    head = f"[*] Running BFS ({args.advance} advance"
    if args.advance == "hybrid":
        head += f", alpha={args.alpha:g}, beta={args.beta:g}"
    print(head + f") from source vertex {src}")
    t0 = time.perf_counter()
    with _Timer() as tm:
        det = b.run(mode, args.alpha, args.beta)
    host_ms = (time.perf_counter() - t0) * 1e3
    print("[!] Done", file=sys.stderr)
    print(f"Iterations: {det.iterations}", file=sys.stderr)
    if args.advance == "hybrid":
        print(f"Push steps: {len(det.push_steps)}", file=sys.stderr)
        print(f"Pull steps: {len(det.pull_steps)}", file=sys.stderr)
        print(_advance_runs(det), file=sys.stderr)
    depth = b.getDistances()
    if args.validate:
        _validate(lambda: np.array_equal(depth, cpu_bfs(csr, src)))
    if args.print:
        print(f"{'Vertex':<10}{'Distance':<10}")
        for v in np.nonzero(depth != csr.n + 1)[0]:
            print(f"{int(v):<10}{int(depth[v]):<10}")
    _profile(args, "bfs_kernel", tm.ms, det.visited_edges, _steps_ms(b.level_records()))
    print(f"Total Host Time: {int(host_ms)} ms")
    return 0


def _advance_runs(det) -> str:
    """The reference's "(push xA, pull xB, ...)" summary of the schedule."""
    pulls = set(det.pull_steps)
    runs, cur, cnt = [], None, 0
    for i in range(det.iterations):
        k = "pull" if i in pulls else "push"
        if k != cur and cnt:
            runs.append(f"{cur} x{cnt}")
            cnt = 0
        cur = k
        cnt += 1
    if cnt:
        runs.append(f"{cur} x{cnt}")
    return "(" + ", ".join(runs) + ")"


def run_sssp(args) -> int:
    from . import algorithms
    csr = _read(args, WEIGHT_F32)
    G = _build(csr)
    s = algorithms.SSSP(G)
    if args.delta:
        s.set_delta(args.delta)
    src = _source(args, csr.n)
    s.init(src)
    print(f"[*] Running SSSP on source {src}")
    t0 = time.perf_counter()
    with _Timer() as tm:
        it = s.run()
    host_ms = (time.perf_counter() - t0) * 1e3
    print("[!] Done", file=sys.stderr)
    print(f"Iterations: {it}", file=sys.stderr)
    dist = s.getDistances()
    if args.validate:
        _validate(lambda: np.array_equal(dist.view(np.uint32), cpu_sssp(csr, src).view(np.uint32)))
    if args.print:
        print(f"{'Vertex':<10}{'Distance':<10}")
        for v in np.nonzero(dist != dist.dtype.type(csr.n + 1))[0]:
            print(f"{int(v):<10}{dist[v]:<10}")
    reached = dist != dist.dtype.type(csr.n + 1)
    edges = int(np.diff(csr.row_offsets.astype(np.int64))[reached].sum())
    _profile(args, "sssp_kernel", tm.ms, edges, _steps_ms(s.level_records()))
    print(f"Total Host Time: {int(host_ms)} ms")
    return 0


def run_cc(args) -> int:
    from . import algorithms
    csr = _read(args, WEIGHT_U32)
    G = _build(csr)
    cc = algorithms.CC(G)
    src = _source(args, csr.n)
    cc.init(src)
    print(f"[*] Running CC on source {src}")
    t0 = time.perf_counter()
    with _Timer() as tm:
        cc.run()
    host_ms = (time.perf_counter() - t0) * 1e3
    print("[!] Done", file=sys.stderr)
    lab = cc.getLabels()
    if args.validate:
        _validate(lambda: np.array_equal(lab, cpu_cc(csr)))
    if args.print:
        print(f"{'Vertex':<10}{'Label':<10}")
        for v in range(csr.n):
            print(f"{v:<10}{int(lab[v]):<10}")
    # union-find on undirected graphs, the reference's propagation on directed ones
    _profile(args, "cc_kernel" if G.properties.directed else "uf_*_kernel", tm.ms, csr.m)
    print(f"Total Host Time: {int(host_ms)} ms")
    return 0


def run_bc(args) -> int:
    from . import algorithms
    csr = _read(args, WEIGHT_U32)
    G = _build(csr)
    bc = algorithms.BC(G)
    src = _source(args, csr.n)
    bc.init(src)
    print(f"[*] Running BC on source {src}")
    t0 = time.perf_counter()
    with _Timer() as tm:
        bc.run()
    host_ms = (time.perf_counter() - t0) * 1e3
    print("[!] Done", file=sys.stderr)
    val = bc.getBC()
    if args.validate:  # float32 on the GPU against float64 here
        ref = cpu_bc(csr, [src])
        _validate(lambda: np.allclose(val, ref, rtol=1e-4, atol=1e-4))
    if args.print:
        print(f"{'Vertex':<10}{'BC':<10}")
        for v in range(csr.n):
            print(f"{v:<10}{val[v]:<10}")
    _profile(args, "bc_kernel", tm.ms, csr.m)
    print(f"Total Host Time: {int(host_ms)} ms")
    return 0


def run_tc(args) -> int:
    from . import algorithms
    csr = _read(args, WEIGHT_U32)
    G = _build(csr)
    tc = algorithms.TC(G)
    tc.init()
    print("[*] Running TC")
    t0 = time.perf_counter()
    with _Timer() as tm:
        tc.run()
    host_ms = (time.perf_counter() - t0) * 1e3
    print("[!] Done", file=sys.stderr)
    if args.validate:
        _validate(lambda: tc.getNumTriangles() == cpu_tc(csr))
    if args.print:
        print(f"Total num triangles: {tc.getNumTriangles()}")
    _profile(args, "tc_hash_kernel", tm.ms, csr.m)
    print(f"Total Host Time: {int(host_ms)} ms")
    return 0


def _read(args, value_type: int) -> CSR:
    print("[*] Reading CSR", file=sys.stderr)
    return read_graph(args, value_type)


def _build(csr: CSR):
    from .core import build
    _device_info()
    print("[*] Building Graph", file=sys.stderr)
    G = build.fromCSR(csr)
    _graph_info(G)
    return G


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="python -m sygraph_b200.cli", description="SYgraph example programs")
    sub = ap.add_subparsers(dest="algorithm", required=True)
    for name in ("bfs", "sssp", "cc", "bc", "tc"):
        p = sub.add_parser(name)
        fmt = p.add_mutually_exclusive_group()
        fmt.add_argument("-b", "--binary", action="store_true", help="Treat input as binary CSR format")
        fmt.add_argument("-m", "--matrix-market", action="store_true", help="Treat input as Matrix Market format")
        p.add_argument("-p", "--print", action="store_true", help="Print algorithm output to stdout")
        prof = p.add_mutually_exclusive_group()
        prof.add_argument("-v", action="store_true", help="Print grouped kernel timing summary")
        prof.add_argument("-V", action="store_true", help="Print detailed timing for each kernel invocation")
        p.add_argument("-c", "--validate", action="store_true",
                       help="Validate algorithm output against CPU implementation")
        p.add_argument("-u", "--undirected", action="store_true", help="Treat input COO as an undirected graph")
        p.add_argument("-s", "--source", type=_nonneg, default=None, help="Specify the source vertex")
        p.add_argument("graph", help="Path to the graph file")
        if name == "bfs":
            p.add_argument("--advance", type=str.lower, choices=["push", "pull", "hybrid"], default="push",
                           help="Select BFS advance strategy (push|pull|hybrid)")
            p.add_argument("--alpha", type=_positive, default=15.0, help="Alpha parameter for hybrid BFS")
            p.add_argument("--beta", type=_positive, default=24.0, help="Beta parameter for hybrid BFS")
        if name == "sssp":
            p.add_argument("--delta", type=float, default=0.0,
                           help="Near-far bucket width (0: the reference's frontier Bellman-Ford)")
    return ap


def _nonneg(x: str) -> int:
    v = int(x)
    if v < 0:
        raise argparse.ArgumentTypeError("must be a non-negative number")
    return v


def _positive(x: str) -> float:
    v = float(x)
    if v <= 0:
        raise argparse.ArgumentTypeError("must be a positive number")
    return v


def main(argv=None) -> int:
    args = parser().parse_args(argv)
    return {"bfs": run_bfs, "sssp": run_sssp, "cc": run_cc, "bc": run_bc, "tc": run_tc}[args.algorithm](args)


if __name__ == "__main__":
    sys.exit(main())
