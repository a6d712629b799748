"""Host side of the example-program front end (sygraph_b200/cli.py): the text
COO reader follows io::coo::fromCOO + io::csr::fromCOO (rows in edge order,
no sorting or de-duplication, n = largest id + 1), the flags follow
examples/include/utils.hpp:41-97, and the CPU checks agree with the oracle."""
import numpy as np
import pytest

from sygraph_b200 import cli


def _write(tmp_path, text):
    p = tmp_path / "g.coo"
    p.write_text(text)
    return str(p)


def test_coo_text_reader_keeps_edge_order(tmp_path):
    path = _write(tmp_path, "% comment\n% another\n4 4 5\n2 0 0.5\n0 3 1.5\n2 1 2.0\n0 1 0.25\n3 3 1\n")
    g = cli.read_coo_text(path)
    assert g.n == 4 and g.m == 5
    assert g.row_offsets.tolist() == [0, 2, 2, 4, 5]
    assert g.column_indices.tolist() == [3, 1, 0, 1, 3]  # file order inside each row
    assert g.values.tolist() == [1.5, 0.25, 0.5, 2.0, 1.0]
    assert g.properties.directed and g.properties.weighted


def test_coo_text_reader_unsigned_weights_take_leading_digits(tmp_path):
    from sygraph_b200.core import WEIGHT_U32
    g = cli.read_coo_text(_write(tmp_path, "2 2 3\n0 1 0.75\n1 0 12.5\n1 1 7\n"), value_type=WEIGHT_U32)
    assert g.values.tolist() == [0, 12, 7]


def test_coo_text_reader_undirected_interleaves_reverse_edges(tmp_path):
    path = _write(tmp_path, "3 3 2\n0 1\n2 0\n")
    g = cli.read_coo_text(path, undirected=True)
    # entries (0,1) (1,0) (2,0) (0,2), counting-sorted by row
    assert g.row_offsets.tolist() == [0, 2, 3, 4]
    assert g.column_indices.tolist() == [1, 2, 0, 0]
    assert g.values is None and not g.properties.directed


def test_flags(tmp_path):
    p = cli.parser()
    a = p.parse_args(["bfs", "-c", "-p", "-v", "-u", "-s", "3", "--advance", "HYBRID", "--alpha", "2", "g"])
    assert a.validate and a.print and a.v and a.undirected and a.source == 3 and a.advance == "hybrid"
    assert a.alpha == 2.0 and a.beta == 24.0
    for bad in (["bfs", "-b", "-m", "g"], ["bfs", "-v", "-V", "g"], ["bfs", "-s", "-1", "g"],
                ["bfs", "--advance", "sideways", "g"], ["bfs", "--alpha", "0", "g"], ["cc"]):
        with pytest.raises(SystemExit):
            p.parse_args(bad)
    assert p.parse_args(["sssp", "--delta", "0.1", "g"]).delta == 0.1


def test_cpu_checks_match_the_oracle(oracle, rmat):
    g = rmat(10, perm_seed=3)
    s = int(np.argmax(g.degrees()))
    assert np.array_equal(cli.cpu_bfs(g, s), oracle.bfs_levels(g, s))
    assert np.array_equal(cli.cpu_sssp(g, s).view(np.uint32), oracle.sssp_dijkstra(g, s).view(np.uint32))
    srcs = [s, 5, 17]
    assert np.allclose(cli.cpu_bc(g, srcs), oracle.bc(g, srcs), rtol=1e-12, atol=1e-9)
    assert cli.cpu_tc(g) == oracle.tc_dag(g)[0]
    lab = cli.cpu_cc(g)
    # on a symmetric graph: the largest id of each component
    for comp in np.unique(lab):
        members = np.nonzero(lab == comp)[0]
        assert members.max() == comp
