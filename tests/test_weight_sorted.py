"""The weight-sorted adjacency of delta-stepping SSSP, built on the device
(sg_graph_weight_sorted): every row holds the same (column, weight) pairs as
the CSR, in non-decreasing weight order with equal weights in column order,
and the symmetry flag is right."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_sorted(g):
    ro, col, val = g.row_offsets, g.column_indices, g.values
    bits = val.view(np.uint32) if val.dtype == np.float32 else val
    rows = np.repeat(np.arange(g.n, dtype=np.uint64), np.diff(ro.astype(np.int64)))
    order = np.lexsort((col, bits, rows))  # by row, then weight, then column
    return col[order], val[order]


@pytest.mark.parametrize("kind", ["rmat_f32", "rmat_u32", "grid_u32", "directed", "asym_weights"])
def test_weight_sorted_rows(sg, rmat, kind):
    props = None
    if kind == "rmat_f32":
        g = rmat(16, perm_seed=3)
    elif kind == "rmat_u32":
        g = rmat(14, value_type=sg.WEIGHT_U32)
    elif kind == "grid_u32":
        g = sg.io.grid(200, 0.02, value_type=sg.WEIGHT_U32)
    else:
        rng = np.random.default_rng(7)
        n, k = 3000, 40000
        s, d = rng.integers(0, n, k), rng.integers(0, n, k)
        w = rng.integers(1, 9, k).astype(np.uint32)
        if kind == "directed":
            g = sg.io.fromCOO(n, s, d, w, dedupe=True, drop_self_loops=True)
            props = sg.Properties(directed=True, weighted=True)
        else:  # symmetric pattern, weights differ by direction
            g = sg.io.fromCOO(n, np.concatenate([s, d]), np.concatenate([d, s]),
                              np.concatenate([w, w + 1]), dedupe=True, drop_self_loops=True)
    G = sg.graph.build.fromCSR(g, props)
    col, val, sym = G.weight_sorted()
    want_col, want_val = host_sorted(g)
    assert np.array_equal(col, want_col)
    assert np.array_equal(val.view(np.uint32), want_val.view(np.uint32))
    assert sym == kind.startswith(("rmat", "grid"))
