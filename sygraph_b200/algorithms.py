"""Algorithm classes with the reference's interface (algorithms/*.hpp):
``BFS(G).init(src); BFS.run(direction, alpha, beta) -> BFSRunDetails;
getDistances()``, and the same shape for SSSP, CC, BC and TC.  Each run is
one fused device-side traversal behind the C ABI."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import call, lib
from .core import WEIGHT_F32, Graph, _ptr


class bfs_direction:  # noqa: N801 - algorithms::bfs_direction (bfs.hpp:29)
    push = 0
    pull = 1
    hybrid = 2
    learned = 3  # not in the reference: the learned selector picks every level's strategy


@dataclass
class BFSRunDetails:
    """algorithms::BFSRunDetails (bfs.hpp:31-35)."""
    iterations: int = 0
    push_steps: set = field(default_factory=set)
    pull_steps: set = field(default_factory=set)
    visited_vertices: int = 0
    visited_edges: int = 0


def _details(d: _lib.BfsDetails) -> BFSRunDetails:
    out = BFSRunDetails(iterations=int(d.iterations), visited_vertices=int(d.visited_vertices),
                        visited_edges=int(d.visited_edges))
    for i in range(min(out.iterations, _lib.SG_MAX_LOGGED_LEVELS)):
        (out.pull_steps if d.step_is_pull[i] else out.push_steps).add(i)
    return out


class BFS:
    """algorithms::BFS (bfs.hpp:120-351)."""

    def __init__(self, G: Graph):
        self.G = G
        h = C.c_void_p()
        call("sg_bfs_create", G.handle, C.byref(h))
        self.handle = h
        self._init = False

    def init(self, source: int) -> None:
        call("sg_bfs_init", self.handle, int(source))
        self._init = True

    def reset(self) -> None:
        call("sg_bfs_reset", self.handle)
        self._init = False

    def run(self, direction: int = bfs_direction.push, alpha: float = 1.0, beta: float = 1.0) -> BFSRunDetails:
        d = _lib.BfsDetails()
        call("sg_bfs_run", self.handle, direction, alpha, beta, C.byref(d))
        return _details(d)

    def run_async(self, direction: int = bfs_direction.push, alpha: float = 1.0, beta: float = 1.0) -> None:
        call("sg_bfs_run_async", self.handle, direction, alpha, beta)

    def getDistances(self) -> np.ndarray:
        out = np.empty(self.G.getVertexCount(), np.uint32)
        call("sg_bfs_get_distances", self.handle, _ptr(out))
        return out

    def getDistance(self, v: int) -> int:
        return int(self.getDistances()[v])

    def set_schedule(self, strategies) -> None:
        """Force the strategy of level i (0..5, -1 = the mode decides)."""
        s = np.ascontiguousarray(strategies if strategies is not None else [], np.int32)
        call("sg_bfs_set_schedule", self.handle, s.ctypes.data_as(C.POINTER(C.c_int)), s.size)

    def set_selector(self, mlp, allowed: int = 0x3F, margin: float | None = None,
                     min_frontier: float | None = None) -> None:
        """The MLP of bfs_direction.learned (None detaches it); `margin` is the
        predicted log-time gain it needs to overrule the heuristic, and
        frontiers below `min_frontier` of the vertices keep the heuristic's
        choice without an inference; the model's graph and frontier ranges
        (mlp.graph_range, mlp.frontier_range) limit it to the graphs and
        levels on which it pays for its inferences in training."""
        self._mlp = mlp  # keep the device parameters alive
        call("sg_bfs_set_selector", self.handle, mlp.handle if mlp is not None else None, allowed)
        rng = getattr(mlp, "graph_range", None) if mlp is not None else None
        lo, hi = rng if rng is not None else (-np.inf, np.inf)
        call("sg_bfs_set_selector_graph_range", self.handle, float(lo), float(hi))
        fr = getattr(mlp, "frontier_range", None) if mlp is not None else None
        if fr is not None:
            call("sg_bfs_set_selector_min_frontier", self.handle, float(fr[0]))
            call("sg_bfs_set_selector_max_frontier", self.handle, float(fr[1]))
        if margin is not None:
            call("sg_bfs_set_selector_margin", self.handle, float(margin))
        if min_frontier is not None:
            call("sg_bfs_set_selector_min_frontier", self.handle, float(min_frontier))

    def set_pull_order(self, reverse_levels: int) -> None:
        """Bit L: level L's pull probes in-neighbours from the back."""
        call("sg_bfs_set_pull_order", self.handle, int(reverse_levels))

    def set_launch(self, max_ctas: int = 0, stream=None) -> None:
        """Persistent grid cap (0: every SM) and stream of this instance."""
        call("sg_bfs_set_launch", self.handle, stream, int(max_ctas))

    def log_features(self, enable: bool = True) -> None:
        call("sg_bfs_log_features", self.handle, int(enable))

    def level_features(self) -> np.ndarray:
        out = np.zeros((_lib.SG_MAX_LOGGED_LEVELS, 12), np.float32)
        cnt = C.c_uint32()
        call("sg_bfs_level_features", self.handle, out.ctypes.data_as(C.POINTER(C.c_float)),
             _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return out[:cnt.value]

    def level_times_us(self) -> np.ndarray:
        return np.array([(r["t_end_ns"] - r["t_start_ns"]) / 1000.0 for r in self.level_records()])

    def level_records(self) -> list[dict]:
        recs = (_lib.LevelRecord * _lib.SG_MAX_LOGGED_LEVELS)()
        cnt = C.c_uint32()
        call("sg_bfs_level_records", self.handle, recs, _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return [{k: getattr(recs[i], k) for k, _ in _lib.LevelRecord._fields_} for i in range(cnt.value)]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_bfs_destroy(h)
            self.handle = None


class MultiBFS:
    """Batched BFS from up to 64 sources in one launch (bit-parallel); depths
    per source equal BFS(G).run from that source."""

    def __init__(self, G: Graph, max_sources: int = 64):
        self.G = G
        h = C.c_void_p()
        call("sg_msbfs_create", G.handle, max_sources, C.byref(h))
        self.handle = h
        self.k = 0
        self.details = None

    def run(self, sources, direction: int = bfs_direction.hybrid, alpha: float = 15.0, beta: float = 24.0):
        src = np.ascontiguousarray(sources, np.uint32)
        d = _lib.MsbfsDetails()
        call("sg_msbfs_run", self.handle, _ptr(src), src.size, direction, alpha, beta, C.byref(d))
        self.k = src.size
        self.details = {k: int(getattr(d, k)) for k, _ in _lib.MsbfsDetails._fields_}
        return self.details

    def run_async(self, sources, direction: int = bfs_direction.hybrid, alpha: float = 15.0,
                  beta: float = 24.0) -> None:
        src = np.ascontiguousarray(sources, np.uint32)
        call("sg_msbfs_run_async", self.handle, _ptr(src), src.size, direction, alpha, beta)
        self.k = src.size

    def level_records(self) -> list[dict]:
        recs = (_lib.LevelRecord * _lib.SG_MAX_LOGGED_LEVELS)()
        cnt = C.c_uint32()
        call("sg_msbfs_level_records", self.handle, recs, _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return [{k: getattr(recs[i], k) for k, _ in _lib.LevelRecord._fields_} for i in range(cnt.value)]

    def set_launch(self, max_ctas: int = 0, stream=None) -> None:
        call("sg_msbfs_set_launch", self.handle, stream, int(max_ctas))

    def set_schedule(self, directions) -> None:
        """Forced direction per level (0 push, 2 pull, -1 the mode decides);
        an empty sequence clears it."""
        d = np.ascontiguousarray(list(directions), np.int32)
        call("sg_msbfs_set_schedule", self.handle, d.ctypes.data_as(C.POINTER(C.c_int)) if d.size else None, d.size)

    def set_selector(self, mlp, margin: float = 0.05) -> None:
        """The MLP of bfs_direction.learned (None detaches it), asked where
        the heuristic would switch direction on frontiers inside the model's
        frontier range (mlp.frontier_range, else every size); `margin` is the
        predicted log-time gain it needs to overrule the heuristic."""
        self._mlp = mlp  # keep the device parameters alive
        fr = getattr(mlp, "frontier_range", None) if mlp is not None else None
        lo, hi = fr if fr is not None else (0.0, 1.0)
        call("sg_msbfs_set_selector", self.handle, mlp.handle if mlp is not None else None, float(margin),
             float(lo), float(hi))

    def log_features(self, enable: bool = True) -> None:
        call("sg_msbfs_log_features", self.handle, int(enable))

    def level_features(self) -> np.ndarray:
        out = np.zeros((_lib.SG_MAX_LOGGED_LEVELS, 12), np.float32)
        cnt = C.c_uint32()
        call("sg_msbfs_level_features", self.handle, out.ctypes.data_as(C.POINTER(C.c_float)),
             _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return out[:cnt.value]

    def level_times_us(self) -> np.ndarray:
        return np.array([(r["t_end_ns"] - r["t_start_ns"]) / 1000.0 for r in self.level_records()])

    def getDistances(self) -> np.ndarray:
        """k x n depths (row s: depths from sources[s])."""
        out = np.empty((self.k, self.G.getVertexCount()), np.uint32)
        call("sg_msbfs_get_depths", self.handle, _ptr(out))
        return out

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_msbfs_destroy(h)
            self.handle = None


class SSSP:
    """algorithms::SSSP (sssp.hpp:109-217)."""

    def __init__(self, G: Graph):
        self.G = G
        h = C.c_void_p()
        call("sg_sssp_create", G.handle, C.byref(h))
        self.handle = h
        self.iterations = 0

    def init(self, source: int) -> None:
        call("sg_sssp_init", self.handle, int(source))

    def run(self) -> int:
        it = C.c_uint64()
        call("sg_sssp_run", self.handle, C.byref(it))
        self.iterations = it.value
        return it.value

    def run_async(self) -> None:
        call("sg_sssp_run_async", self.handle)

    def level_records(self) -> list[dict]:
        recs = (_lib.LevelRecord * _lib.SG_MAX_LOGGED_LEVELS)()
        cnt = C.c_uint32()
        call("sg_sssp_level_records", self.handle, recs, _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return [{k: getattr(recs[i], k) for k, _ in _lib.LevelRecord._fields_} for i in range(cnt.value)]

    def set_pull(self, ratio: int) -> None:
        """Pull iterations when frontier out-degree * ratio > m (0: push only)."""
        call("sg_sssp_set_pull", self.handle, int(ratio))

    def set_launch(self, max_ctas: int = 0, stream=None) -> None:
        call("sg_sssp_set_launch", self.handle, stream, int(max_ctas))

    def set_delta(self, delta: float) -> None:
        """Near-far threshold step (0: the reference's frontier Bellman-Ford)."""
        call("sg_sssp_set_delta", self.handle, float(delta))

    def set_tail(self, fraction: float) -> None:
        """Near-far: once fewer than fraction * n vertices wait beyond the
        threshold, finish with plain Bellman-Ford (0: bucket to the end)."""
        call("sg_sssp_set_tail", self.handle, float(fraction))

    def set_heavy_pull(self, ratio: int) -> None:
        """Near-far on symmetric weighted graphs: a bucket's heavy edges go by
        pull when they number more than m / ratio (0: always push)."""
        call("sg_sssp_set_heavy_pull", self.handle, int(ratio))

    def set_selector(self, mlp, margin: float = 0.05) -> None:
        """The MLP that chooses push or pull for the heavy phases of
        delta-stepping (None detaches it), asked on buckets whose heavy edges
        are within the model's heavy range (mlp.heavy_range, a fraction of m;
        else every bucket); `margin` is the predicted log-time gain it needs
        to overrule the heavy_pull rule."""
        self._mlp = mlp  # keep the device parameters alive
        hr = getattr(mlp, "heavy_range", None) if mlp is not None else None
        lo, hi = hr if hr is not None else (0.0, 1e30)
        call("sg_sssp_set_selector", self.handle, mlp.handle if mlp is not None else None, float(margin),
             float(lo), float(hi))

    def log_features(self, enable: bool = True) -> None:
        call("sg_sssp_log_features", self.handle, int(enable))

    def level_features(self) -> np.ndarray:
        """Twelve features per heavy phase of the last run."""
        out = np.zeros((_lib.SG_MAX_LOGGED_LEVELS, 12), np.float32)
        cnt = C.c_uint32()
        call("sg_sssp_level_features", self.handle, out.ctypes.data_as(C.POINTER(C.c_float)),
             _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return out[:cnt.value]

    def set_light_pull(self, ratio: int) -> None:
        """Near-far on symmetric weighted graphs: an iteration whose frontier
        holds more than n / ratio vertices relaxes light edges by pull (0:
        always push)."""
        call("sg_sssp_set_light_pull", self.handle, int(ratio))

    def getDistances(self) -> np.ndarray:
        dt = np.float32 if self.G.value_type == WEIGHT_F32 else np.uint32
        out = np.empty(self.G.getVertexCount(), dt)
        call("sg_sssp_get_distances", self.handle, C.c_void_p(out.ctypes.data))
        return out

    def getDistance(self, v: int):
        return self.getDistances()[v]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_sssp_destroy(h)
            self.handle = None


class CC:
    """algorithms::CC (cc.hpp:74-192): labels[v] = max id over the vertices reaching v.
    The instance owns the labels and the engine workspace, so runs allocate nothing."""

    def __init__(self, G: Graph):
        self.G = G
        h = C.c_void_p()
        call("sg_cc_create", G.handle, C.byref(h))
        self.handle = h
        self.iterations = 0
        self._labels = None

    def init(self, source: int = 0) -> None:
        self.source = source

    def run(self) -> None:
        it = C.c_uint64()
        call("sg_cc_run", self.handle, C.byref(it))
        self.iterations = it.value
        self._labels = None

    def run_async(self) -> None:
        """Enqueue a run on the graph's stream; getLabels() waits for it."""
        call("sg_cc_run_async", self.handle)
        self._labels = None

    AUTO, PROPAGATION, UNION_FIND = 0, 1, 2

    def set_method(self, method: int) -> None:
        """AUTO (union-find on undirected graphs), PROPAGATION (the reference's
        maximum-label propagation) or UNION_FIND; the labels are the same."""
        call("sg_cc_set_method", self.handle, int(method))

    def getLabels(self) -> np.ndarray:
        if self._labels is None:
            out = np.empty(self.G.getVertexCount(), np.uint32)
            call("sg_cc_get_labels", self.handle, _ptr(out))
            self._labels = out
        return self._labels

    labels = property(getLabels)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_cc_destroy(h)
            self.handle = None


class BC:
    """algorithms::BC (bc.hpp:274-419); init accepts one source or a list."""

    def __init__(self, G: Graph):
        self.G = G
        self.sources = None
        self.values = None

    def init(self, source) -> None:
        self.sources = np.atleast_1d(np.asarray(source, dtype=np.uint32))

    def run(self) -> None:
        self.values = np.empty(self.G.getVertexCount(), np.float32)
        call("sg_bc", self.G.handle, _ptr(self.sources), self.sources.size, self.values.ctypes.data_as(
            C.POINTER(C.c_float)))

    def getBC(self) -> np.ndarray:
        return self.values


class BatchedBC:
    """Brandes BC with up to 64 sources per launch (bit-parallel frontiers);
    getBC() equals BC(G) over the same sources within float32 rounding, and
    repeated runs give identical bits."""

    def __init__(self, G: Graph, history_levels: int = 0):
        self.G = G
        h = C.c_void_p()
        call("sg_bc_batch_create", G.handle, history_levels, C.byref(h))
        self.handle = h
        self.details = None

    def run(self, sources, accumulate: bool = False) -> dict:
        """Sources in batches of 64; the first batch overwrites unless `accumulate`."""
        src = np.ascontiguousarray(np.atleast_1d(sources), np.uint32)
        tot = {"iterations": 0, "reached_edges": 0, "history_levels": 0, "history_retries": 0}
        for i in range(0, src.size, 64):
            part = np.ascontiguousarray(src[i:i + 64])
            d = _lib.BcBatchDetails()
            call("sg_bc_batch_run", self.handle, _ptr(part), part.size, int(accumulate or i > 0), C.byref(d))
            tot["iterations"] = max(tot["iterations"], int(d.iterations))
            tot["reached_edges"] += int(d.reached_edges)
            tot["history_levels"] = int(d.history_levels)
            tot["history_retries"] += int(d.history_retries)
        self.details = tot
        return tot

    def run_async(self, sources, accumulate: bool = False) -> None:
        src = np.ascontiguousarray(np.atleast_1d(sources), np.uint32)
        assert src.size <= 64
        call("sg_bc_batch_run_async", self.handle, _ptr(src), src.size, int(accumulate))

    def getBC(self) -> np.ndarray:
        out = np.empty(self.G.getVertexCount(), np.float32)
        call("sg_bc_batch_get", self.handle, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def set_launch(self, max_ctas: int = 0, stream=None) -> None:
        call("sg_bc_batch_set_launch", self.handle, stream, int(max_ctas))

    def level_records(self) -> list[dict]:
        recs = (_lib.LevelRecord * _lib.SG_MAX_LOGGED_LEVELS)()
        cnt = C.c_uint32()
        call("sg_bc_batch_level_records", self.handle, recs, _lib.SG_MAX_LOGGED_LEVELS, C.byref(cnt))
        return [{k: getattr(recs[i], k) for k, _ in _lib.LevelRecord._fields_} for i in range(cnt.value)]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_bc_batch_destroy(h)
            self.handle = None


class TC:
    """algorithms::TC (tc.hpp:473-565), exact.  The instance owns the DAG and
    the work lists, so runs allocate nothing."""

    def __init__(self, G: Graph):
        self.G = G
        h = C.c_void_p()
        call("sg_tc_create", G.handle, C.byref(h))
        self.handle = h
        self.total = None
        self.per_vertex = None

    def init(self) -> None:
        self.total = None

    def run(self, per_vertex: bool = False) -> None:
        tot = C.c_uint64()
        call("sg_tc_run", self.handle, int(per_vertex), C.byref(tot))
        self.total = tot.value
        self.per_vertex = None
        if per_vertex:
            pv = np.zeros(self.G.getVertexCount(), np.uint64)
            call("sg_tc_get_per_vertex", self.handle, pv.ctypes.data_as(C.POINTER(C.c_uint64)))
            self.per_vertex = pv

    def run_async(self, per_vertex: bool = False) -> None:
        """Enqueue a run on the graph's stream; getNumTriangles() waits for it."""
        call("sg_tc_run_async", self.handle, int(per_vertex))
        self.total = None

    def set_shorter_rows(self, shorter: bool = True) -> None:
        """True (default): each DAG edge streams its shorter row; False: the head's row."""
        call("sg_tc_set_shorter_rows", self.handle, int(shorter))

    def getNumTriangles(self, v: int | None = None) -> int:
        if v is None:
            if self.total is None:
                tot = C.c_uint64()
                call("sg_tc_get_total", self.handle, C.byref(tot))
                self.total = tot.value
            return int(self.total)
        if self.per_vertex is None:
            self.run(per_vertex=True)
        return int(self.per_vertex[v])

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_tc_destroy(h)
            self.handle = None
