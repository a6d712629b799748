"""What the trained selector gains over the reference heuristic, on per-level
cost tables measured on a B200 for held-out graphs (RMAT-22 with another
seed, RMAT-23, a 4096x4096 grid with long-range pairs, a uniform random
graph).  The fixture was made by
`python -m sygraph_b200.train_selector collect --set eval --out tests/golden/selector_eval_b200.npz`
and the model by `... train`; the schedules here come from the FP64 oracle
forward pass of the committed parameters, replaying the engine's rule
(MLP argmin inside the trusted range and the model's graph and frontier
ranges, heuristic outside them)."""
import numpy as np
import pytest

from conftest import ROOT

EVAL = ROOT / "tests" / "golden" / "selector_eval_b200.npz"
MODEL = ROOT / "sygraph_b200" / "models" / "selector_b200.npz"
# level-time tables of the training graphs (`train_selector collect --set
# train`, kept without the per-sample arrays: T, H, F0, offsets, names)
TRAIN_TABLES = ROOT / "tests" / "golden" / "selector_train_tables_b200.npz"


@pytest.fixture(scope="module")
def tables():
    from sygraph_b200 import train_selector as ts
    with np.load(EVAL) as d:
        data = {k: d[k] for k in d.files}
    with np.load(MODEL) as m:
        params = m["params"].astype(np.float32)
        gates = {"graph_range": tuple(m["graph_range"]), "frontier_range": tuple(m["frontier_range"])}
    return ts, data, params, gates


def _schedules(ts, data, params, gates):
    from oracle import mlp as omlp
    fwd = lambda X: omlp.forward(params.astype(np.float64), X)[0]  # noqa: E731
    lo, hi = gates["frontier_range"]
    out = []
    for name, T, H, F in ts.traversals(data):
        c = ts.simulate_choices(params, fwd, F, H, graph_range=gates["graph_range"], min_frontier=lo,
                                max_frontier=hi)
        idx = np.arange(len(T))
        out.append((name, T[idx, H].sum(), T[idx, c].sum(), T.min(1).sum(), c, H))
    return out


def test_model_file_layout(tables):
    ts, _, params, gates = tables
    g0, g1 = gates["graph_range"]
    f0, f1 = gates["frontier_range"]
    assert g0 < g1 and 0.0 <= f0 < f1 <= 1.0
    from oracle import mlp as omlp
    assert params.size == sum(int(np.prod(s)) for _, s in omlp.SHAPES)
    t = params.size - 48
    lo, hi = params[t + 24:t + 36], params[t + 36:t + 48]
    assert np.all(lo < hi) and np.all(np.isfinite(params))


def test_learned_schedule_beats_heuristic_on_held_out_graphs(tables):
    ts, data, params, gates = tables
    rows = _schedules(ts, data, params, gates)
    heur = sum(r[1] for r in rows)
    learned = sum(r[2] for r in rows)
    best = sum(r[3] for r in rows)
    # the whole held-out set: at least 8% less time than the heuristic
    # (the gain is on the grid), within 2% of the per-level best
    assert learned <= 0.92 * heur, (learned, heur)
    assert learned <= 1.02 * best, (learned, best)
    # no traversal more than 6% slower than under the heuristic
    for name, h, l, _, _, _ in rows:
        assert l <= 1.06 * h, (name, l, h)


def test_learned_schedule_on_rmat_is_no_worse_than_heuristic(tables):
    ts, data, params, gates = tables
    rows = [r for r in _schedules(ts, data, params, gates) if r[0].startswith("rmat")]
    assert rows
    heur = sum(r[1] for r in rows)
    learned = sum(r[2] for r in rows)
    assert learned <= 1.03 * heur


def test_regret_bookkeeping_matches_tables(tables):
    """Heuristic schedules in the fixture are the reference's push/pull
    choices (strategy 0 or 2 only) and cover every level."""
    ts, data, _, _ = tables
    for name, T, H, F in ts.traversals(data):
        assert T.shape[1] == 6 and len(H) == len(T) == len(F)
        assert set(np.unique(H)) <= {0, 2}
        assert np.all(T > 0)


class _CpuModel:
    """The committed parameters with the FP64 oracle forward pass, in the
    shape the trainer's gate functions read."""

    def __init__(self, params, graph_range=None, frontier_range=None):
        self.params = params
        self.graph_range = graph_range
        self.frontier_range = frontier_range

    def forward(self, X):
        from oracle import mlp as omlp
        return omlp.forward(self.params.astype(np.float64), np.asarray(X, np.float64))[0]


def test_gates_follow_from_training_tables(tables):
    """The committed frontier and graph ranges are the ones the trainer
    derives from the training tables at the measured inference cost: the
    model is consulted on the grids with long-range pairs, where its choices
    save more than the inferences cost, and on no RMAT graph, where the
    heuristic's switch points were already as good."""
    ts, _, params, gates = tables
    with np.load(TRAIN_TABLES) as d:
        data = {k: d[k] for k in d.files}
    m = _CpuModel(params)
    fr = ts.frontier_range(m, data)
    m.frontier_range = fr
    gr = ts.graph_range(m, data)
    assert np.allclose(fr, gates["frontier_range"], atol=1e-6), (fr, gates)
    assert np.allclose(gr, gates["graph_range"], atol=1e-6), (gr, gates)
    lo, hi = gr
    f9 = {str(n).split(":")[0]: float(F[0][9]) for n, _, _, F in ts.traversals(data)}
    assert all(lo <= v <= hi for k, v in f9.items() if k.startswith("grid") and k != "grid512")
    assert not any(lo <= v <= hi for k, v in f9.items() if k.startswith(("rmat", "uniform")))


# The batched (64-source) BFS's selector: push or pull per level, measured on
# batches of 64 sources of the same held-out graphs
# (`train_selector collect --batched --set eval`), the batched heuristic
# (alpha 4, beta 24) as its fallback.
BATCH_EVAL = ROOT / "tests" / "golden" / "selector_msbfs_eval_b200.npz"
BATCH_TRAIN_TABLES = ROOT / "tests" / "golden" / "selector_msbfs_train_tables_b200.npz"
BATCH_MODEL = ROOT / "sygraph_b200" / "models" / "selector_msbfs_b200.npz"


def _batched_model():
    with np.load(BATCH_MODEL) as m:
        return m["params"].astype(np.float32), tuple(float(x) for x in m["frontier_range"])


def test_batched_learned_schedule_on_held_out_graphs():
    from sygraph_b200 import train_selector as ts
    with np.load(BATCH_EVAL) as d:
        data = {k: d[k] for k in d.files}
    params, (lo, hi) = _batched_model()
    m = _CpuModel(params, None, (lo, hi))
    heur = learned = 0.0
    for name, T, H, F in ts.traversals(data):
        assert set(np.unique(H)) <= {0, 2}
        c = ts.simulate_choices(params, m.forward, F, H, ts.BATCH_ALLOWED, min_frontier=lo, max_frontier=hi,
                                alpha=ts.BATCH_ALPHA, beta=ts.BATCH_BETA)
        assert set(np.unique(c)) <= {0, 2}  # push or pull only
        idx = np.arange(len(T))
        h = float(T[idx, H].sum())
        l = float(T[idx, c].sum()) + ts.INFERENCE_US * int(ts.consulted(F, c, lo, hi, ts.BATCH_ALPHA,
                                                                           ts.BATCH_BETA).sum())
        assert l <= 1.01 * h, (name, l, h)  # no batch more than 1% slower
        heur += h
        learned += l
    assert learned <= heur / 1.02, (learned, heur)  # at least 2% less time over the held-out batches


def test_batched_frontier_range_follows_from_training_tables():
    from sygraph_b200 import train_selector as ts
    with np.load(BATCH_TRAIN_TABLES) as d:
        data = {k: d[k] for k in d.files}
    params, fr = _batched_model()
    got = ts.frontier_range(_CpuModel(params), data, allowed=ts.BATCH_ALLOWED, alpha=ts.BATCH_ALPHA,
                            beta=ts.BATCH_BETA)
    assert np.allclose(got, fr, atol=1e-6), (got, fr)


# Delta-stepping SSSP's selector: push or pull for a bucket's heavy phase,
# per-phase cost tables of the held-out graphs (`train_selector collect --sssp
# --set eval`) and of the training graphs (`--set train`).
SSSP_EVAL = ROOT / "tests" / "golden" / "selector_sssp_eval_b200.npz"
SSSP_TRAIN_TABLES = ROOT / "tests" / "golden" / "selector_sssp_train_tables_b200.npz"
SSSP_MODEL = ROOT / "sygraph_b200" / "models" / "selector_sssp_b200.npz"


def _sssp_model():
    with np.load(SSSP_MODEL) as m:
        params = m["params"].astype(np.float32)
        hr = tuple(float(x) for x in m["heavy_range"])
    mdl = _CpuModel(params)
    mdl.heavy_range = hr
    return mdl


def test_sssp_learned_heavy_phases_on_held_out_graphs():
    """Inference cost included, the model's heavy phases take less time than
    the rule's on the held-out graphs; no source loses more than 1%."""
    from sygraph_b200 import train_selector as ts
    with np.load(SSSP_EVAL) as d:
        data = {k: d[k] for k in d.files}
    rep = ts.evaluate_sssp(_sssp_model(), data)
    assert rep["total"]["learned_us"] <= rep["total"]["heuristic_us"] / 1.01, rep["total"]
    for r in rep["traversals"]:
        assert r["learned_us"] <= 1.01 * r["heuristic_us"] + 2 * ts.INFERENCE_US, r


def test_sssp_heavy_range_follows_from_training_tables():
    from sygraph_b200 import train_selector as ts
    with np.load(SSSP_TRAIN_TABLES) as d:
        data = {k: d[k] for k in d.files}
    mdl = _sssp_model()
    got = ts.heavy_range(mdl, data)
    assert np.allclose(got, mdl.heavy_range, atol=1e-6), (got, mdl.heavy_range)
