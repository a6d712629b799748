"""The example-program front end on the GPU: every algorithm with -c passes
its CPU check on a text COO file, a Matrix Market file and a binary CSR, and
-v / -V / -p print the reference's summary lines."""
import numpy as np
import pytest

from sygraph_b200 import cli

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def coo_file(tmp_path_factory, rmat):
    g = rmat(10, perm_seed=3)
    src = np.repeat(np.arange(g.n), np.diff(g.row_offsets))
    keep = src < g.column_indices
    path = tmp_path_factory.mktemp("cli") / "g.coo"
    with open(path, "w") as f:
        f.write("% rmat-10, one direction of each pair\n")
        f.write(f"{g.n} {g.n} {int(keep.sum())}\n")
        for u, v, w in zip(src[keep], g.column_indices[keep], g.values[keep]):
            f.write(f"{u} {v} {float(w)!r}\n")
    return str(path), g


@pytest.mark.parametrize("algo,extra", [("bfs", ["--advance", "hybrid"]), ("bfs", ["--advance", "pull"]),
                                        ("sssp", []), ("sssp", ["--delta", "0.1"]), ("cc", []), ("bc", []),
                                        ("tc", [])])
def test_every_algorithm_validates(capsys, coo_file, algo, extra):
    path, g = coo_file
    s = str(int(np.argmax(g.degrees())))
    assert cli.main([algo, "-u", "-c", "-v", "-s", s, *extra, path]) == 0
    out = capsys.readouterr().out
    assert "Validation: [Success]" in out, out
    assert "Total GPU Time:" in out and "Total Edge-Througput (MTEPS):" in out and "Total Host Time:" in out


def test_detailed_timing_and_print(capsys, coo_file):
    path, g = coo_file
    assert cli.main(["bfs", "-u", "-V", "-p", "-s", "0", "--advance", "hybrid", path]) == 0
    out = capsys.readouterr().out
    assert "Kernel [bfs_kernel x 1] (0) " in out
    lines = [ln for ln in out.splitlines() if ln[:1].isdigit()]
    assert len(lines) == int((cli.cpu_bfs(cli.read_coo_text(path, True), 0) != g.n + 1).sum())


def test_binary_and_matrix_market_inputs(capsys, tmp_path, rmat):
    import sygraph_b200 as sg
    g = rmat(9, perm_seed=2)
    sg.io.toBinary(g, str(tmp_path / "g.bin"))
    assert cli.main(["bfs", "-b", "-c", "-s", "1", str(tmp_path / "g.bin")]) == 0
    src = np.repeat(np.arange(g.n), np.diff(g.row_offsets))
    keep = src <= g.column_indices
    with open(tmp_path / "g.mtx", "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{g.n} {g.n} {int(keep.sum())}\n")
        for u, v, w in zip(src[keep], g.column_indices[keep], g.values[keep]):
            f.write(f"{v + 1} {u + 1} {float(w)!r}\n")
    assert cli.main(["sssp", "-m", "-c", "-s", "1", str(tmp_path / "g.mtx")]) == 0
    out = capsys.readouterr().out
    assert out.count("Validation: [Success]") == 2, out
