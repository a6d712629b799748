"""The grid barrier of the fused engines never waits without bound: when a
block does not arrive, every other block gives up after its poll limit,
records the timeout in the barrier's error word (what the engines report as
SG_ERR_TIMEOUT) and returns; the context stays usable."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(sg, blocks, skip, limit):
    t, e = C.c_uint32(), C.c_uint32()
    sg._lib.call("sg_debug_barrier_check", blocks, skip, limit, C.byref(t), C.byref(e))
    return t.value, e.value


def test_every_block_arrives(sg):
    assert _check(sg, 16, 16, 1 << 16) == (0, 0)
    assert _check(sg, 1, 1, 1) == (0, 0)


def test_missing_block_times_every_other_block_out(sg, oracle, rmat):
    assert _check(sg, 16, 5, 20000) == (15, 1)
    assert _check(sg, 8, 0, 1) == (7, 1)
    # the context survives: a traversal afterwards is exact
    g = rmat(12, perm_seed=2)
    bfs = sg.algorithms.BFS(sg.graph.build.fromCSR(g))
    s = int(np.argmax(g.degrees()))
    bfs.init(s)
    bfs.run(sg.algorithms.bfs_direction.hybrid, 15.0, 24.0)
    assert np.array_equal(bfs.getDistances(), oracle.bfs_levels(g, s))


def test_argument_checks(sg):
    for args in ((0, 0, 100), (65, 0, 100), (4, 0, 0), (4, 0, (1 << 20) + 1)):
        with pytest.raises(sg._lib.SygraphError):
            _check(sg, *args)
