"""Learned strategy selector: the MLP handle, its training on the GPU, and
the per-level training data the traversal engine generates for itself.

Strategies (the MLP's six outputs): 0 push/warp, 1 push/CTA, 2 pull/warp,
3 pull/CTA, 4 pull_all/warp, 5 pull_all/CTA.  Features (twelve, computed on
the device at every level end, the same way for training and inference):
log and linear frontier size, log and linear frontier degree, unexplored
degree fraction, unvisited fraction, the level-0 and summary bitmap occupancy
a frontier of that size would have if spread at random, mean frontier
degree, graph mean degree, current direction, frontier growth."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from ._lib import call, lib
from .core import DeviceArray

IN, HID, OUT = 12, 32, 6
STRATEGIES = ["push/warp", "push/cta", "pull/warp", "pull/cta", "pull_all/warp", "pull_all/cta"]
MODEL_PATH = Path(__file__).resolve().parent / "models" / "selector_b200.npz"

PARAM_COUNT = int(lib.sg_mlp_param_count())
TRAINABLE_COUNT = HID * IN + HID + HID * HID + HID + OUT * HID + OUT


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """Device-resident MLP (sg_mlp)."""

    def __init__(self, params: np.ndarray | None = None, graph_range=None, frontier_range=None, heavy_range=None):
        # (lo, hi) of the mean-degree feature log2(1 + m/n) / 8 on which the
        # model is consulted (None: every graph); see sg_bfs_set_selector_graph_range
        self.graph_range = None if graph_range is None else (float(graph_range[0]), float(graph_range[1]))
        # (lo, hi) of the frontier size, as a fraction of n, on which it is
        # consulted (None: the engine's defaults); see sg_bfs_set_selector_*_frontier
        self.frontier_range = None if frontier_range is None else (float(frontier_range[0]),
                                                                   float(frontier_range[1]))
        # SSSP heavy phases: (lo, hi) of the bucket's heavy edges as a
        # fraction of m on which the model is consulted; see sg_sssp_set_selector
        self.heavy_range = None if heavy_range is None else (float(heavy_range[0]), float(heavy_range[1]))
        h = C.c_void_p()
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        call("sg_mlp_create", None if p is None else _fptr(p), C.byref(h))
        self.handle = h

    @property
    def params(self) -> np.ndarray:
        out = np.empty(PARAM_COUNT, np.float32)
        call("sg_mlp_get_params", self.handle, _fptr(out))
        return out

    @params.setter
    def params(self, value) -> None:
        v = np.ascontiguousarray(value, np.float32)
        assert v.size == PARAM_COUNT
        call("sg_mlp_set_params", self.handle, _fptr(v))

    def set_normalisation(self, X: np.ndarray, margin: float = 0.25) -> None:
        """Standardise inputs with X's statistics; the trusted range is X's
        range widened by `margin` of its span."""
        p = self.params
        t = TRAINABLE_COUNT
        mean, std = X.mean(0), X.std(0)
        std[std < 1e-6] = 1.0
        lo, hi = X.min(0), X.max(0)
        span = np.maximum(hi - lo, 1e-3)
        p[t:t + IN] = mean
        p[t + IN:t + 2 * IN] = 1.0 / std
        p[t + 2 * IN:t + 3 * IN] = lo - margin * span
        p[t + 3 * IN:t + 4 * IN] = hi + margin * span
        self.params = p

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        dx = DeviceArray(X)
        dy = DeviceArray(shape=(X.shape[0], OUT), dtype=np.float32)
        call("sg_mlp_forward", self.handle, C.c_void_p(dx.ptr), X.shape[0], C.c_void_p(dy.ptr))
        return dy.numpy()

    def gradient(self, X, T, M):
        X, T, M = (np.ascontiguousarray(a, np.float32) for a in (X, T, M))
        dx, dt, dm = DeviceArray(X), DeviceArray(T), DeviceArray(M)
        g = np.empty(PARAM_COUNT, np.float32)
        loss = C.c_float()
        call("sg_mlp_gradient", self.handle, C.c_void_p(dx.ptr), C.c_void_p(dt.ptr), C.c_void_p(dm.ptr), X.shape[0],
             _fptr(g), C.byref(loss))
        return loss.value, g

    def train(self, X, T, M, steps: int = 2000, lr: float = 3e-3, weight_decay: float = 1e-5) -> float:
        X, T, M = (np.ascontiguousarray(a, np.float32) for a in (X, T, M))
        dx, dt, dm = DeviceArray(X), DeviceArray(T), DeviceArray(M)
        loss = C.c_float()
        call("sg_mlp_train", self.handle, C.c_void_p(dx.ptr), C.c_void_p(dt.ptr), C.c_void_p(dm.ptr), X.shape[0],
             steps, lr, weight_decay, C.byref(loss))
        return loss.value

    def choose(self, X: np.ndarray, allowed: int = 0x3F) -> np.ndarray:
        y = self.forward(X)
        y[:, [j for j in range(OUT) if not (allowed >> j) & 1]] = np.inf
        return y.argmin(1)

    def save(self, path=MODEL_PATH, **meta) -> None:
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        if self.graph_range is not None:
            meta["graph_range"] = np.asarray(self.graph_range, np.float32)
        if self.frontier_range is not None:
            meta["frontier_range"] = np.asarray(self.frontier_range, np.float32)
        if self.heavy_range is not None:
            meta["heavy_range"] = np.asarray(self.heavy_range, np.float32)
        np.savez(path, params=self.params, **meta)

    @staticmethod
    def load(path=MODEL_PATH) -> "Mlp":
        d = np.load(path)
        return Mlp(d["params"], d["graph_range"] if "graph_range" in d.files else None,
                   d["frontier_range"] if "frontier_range" in d.files else None,
                   d["heavy_range"] if "heavy_range" in d.files else None)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.sg_mlp_destroy(h)
            self.handle = None
