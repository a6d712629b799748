"""The trainer's replay of the engines' decision rules, on small synthetic
cost tables (no GPU): the heuristic's choice from the features, where the
model is asked (switch points, frontier and graph ranges, the SSSP heavy
range), the margin, and the gates chosen from the tables."""
import numpy as np
import pytest

from sygraph_b200 import train_selector as ts

IN, OUT = 12, 6


class _Table:
    """A model whose prediction is a fixed table lookup by level index
    (feature 0 carries the index), with every feature trusted."""

    def __init__(self, y):
        self.y = np.asarray(y, np.float64)
        n = 1718
        self.params = np.zeros(n, np.float32)
        t = n - 4 * IN
        self.params[t + 2 * IN:t + 3 * IN] = -1e9
        self.params[t + 3 * IN:t + 4 * IN] = 1e9
        self.graph_range = None
        self.frontier_range = None
        self.heavy_range = None

    def forward(self, X):
        return self.y[np.asarray(X)[:, 0].astype(int)]


def _features(levels, f1, f3, f4, f9=0.3):
    F = np.zeros((levels, IN), np.float32)
    F[:, 0] = np.arange(levels)
    F[:, 1] = f1
    F[:, 3] = f3
    F[:, 4] = f4
    F[:, 9] = f9
    return F


def test_heuristic_choice_is_the_reference_rule():
    f = np.zeros(IN, np.float32)
    f[3], f[4], f[1] = 0.2, 1.0, 0.5
    assert ts.heuristic_choice(f, 0, alpha=15.0) == 2  # 0.2 > 1/15: push turns to pull
    assert ts.heuristic_choice(f, 0, alpha=4.0) == 0   # 0.2 < 1/4: stays in push
    assert ts.heuristic_choice(f, 2, beta=24.0) == 2   # 0.5 >= 1/24: stays in pull
    f[1] = 0.01
    assert ts.heuristic_choice(f, 2, beta=24.0) == 0   # below n / beta: back to push


def test_model_is_asked_only_at_switch_points_inside_the_ranges():
    # levels: push, then the heuristic would pull at level 1 (f3 large), stay
    # in pull at level 2, and return to push at level 3 (f1 small)
    F = _features(4, f1=[0.001, 0.1, 0.2, 0.001], f3=[0.0, 0.5, 0.5, 0.5], f4=[1.0, 1.0, 1.0, 1.0])
    H = np.array([0, 2, 2, 0])
    # the model prefers push/warp (0) everywhere, by a wide margin
    y = np.tile([0.0, 9, 5.0, 9, 9, 9], (4, 1))
    m = _Table(y)
    c = ts.simulate_choices(m.params, m.forward, F, H, min_frontier=0.0)
    # asked at level 1 (switch to pull): overrules to push; from push the
    # heuristic would pull again at levels 2 and 3: asked again each time,
    # push again
    assert list(c) == [0, 0, 0, 0]
    asked = ts.consulted(F, c, 0.0, 1.0)
    assert list(asked) == [False, True, True, True]
    # a frontier range that excludes level 1 leaves it to the heuristic
    c2 = ts.simulate_choices(m.params, m.forward, F, H, min_frontier=0.15, max_frontier=1.0)
    assert c2[1] == 2
    # outside the graph range the heuristic decides every level
    c3 = ts.simulate_choices(m.params, m.forward, F, H, min_frontier=0.0, graph_range=(0.5, 0.6))
    assert list(c3) == [0, 2, 2, 0]
    # a margin wider than the predicted gain keeps the heuristic's choice
    c4 = ts.simulate_choices(m.params, m.forward, F, H, min_frontier=0.0, margin=10.0)
    assert list(c4) == [0, 2, 2, 0]


def test_gates_trade_gains_against_inference_cost():
    # one traversal where overruling the switch saves 50 us, one where the
    # model agrees with the heuristic (its inference is pure cost)
    F = _features(3, f1=[0.001, 0.1, 0.1], f3=[0.0, 0.5, 0.0], f4=[1.0, 1.0, 1.0])
    T_gain = np.array([[10, 10, 10, 10, 10, 10], [20, 99, 70, 99, 99, 99], [10, 10, 10, 10, 10, 10]], np.float32)
    data = {"T": np.concatenate([T_gain, T_gain]), "H": np.array([0, 2, 0, 0, 2, 0], np.int32),
            "F0": np.concatenate([F, F]), "offsets": np.array([0, 3, 6]), "names": np.array(["g:1", "g:2"])}
    m = _Table(np.tile([0.0, 9, 5.0, 9, 9, 9], (3, 1)))
    assert ts.frontier_range(m, data, cost_us=2.0) is not None
    m.frontier_range = ts.frontier_range(m, data, cost_us=2.0)
    assert ts.graph_range(m, data, cost_us=2.0) == pytest.approx((0.25, 0.35))
    # an inference cost above the gain closes the graph range
    assert ts.graph_range(m, data, cost_us=1000.0) == (1.0, 0.0)
    rep = ts.evaluate(m, data, cost_us=2.0)["total"]
    assert rep["learned_us"] < rep["heuristic_us"]


def test_sssp_heavy_phase_replay_and_range():
    # three heavy phases; the rule pulls phase 1 (heavy edges 0.2 m) where
    # push is cheaper; phases 0 and 2 are far from the rule's threshold
    F = _features(3, f1=0.1, f3=[0.001, 0.2, 0.9], f4=1.0)
    H = np.array([0, 2, 2], np.int32)
    T = np.array([[5, 9, 50, 9, 9, 9], [60, 99, 100, 99, 99, 99], [300, 999, 100, 999, 999, 999]], np.float32)
    y = np.log(T.astype(np.float64))
    m = _Table(y)
    c = ts.simulate_sssp(m.params, m.forward, F, H, margin=0.05)
    assert list(c) == [0, 0, 2]
    assert list(ts.simulate_sssp(m.params, m.forward, F, H, heavy_range=(0.5, 1.0))) == [0, 2, 2]
    data = {"T": T, "H": H, "F0": F, "offsets": np.array([0, 3]), "names": np.array(["g:1"])}
    hr = ts.heavy_range(m, data, cost_us=2.0)
    assert hr[0] <= 0.2 <= hr[1] and not (hr[0] <= 0.001)
    m.heavy_range = hr
    rep = ts.evaluate_sssp(m, data, cost_us=2.0)["total"]
    assert rep["learned_us"] == pytest.approx(5 + 60 + 100 + 2.0 * rep["inferences"])
    assert rep["heuristic_us"] == pytest.approx(5 + 100 + 100)
