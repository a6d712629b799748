"""Extract the reference's known-answer fixtures into tests/golden/kat.json.

Reads SYgraph's test sources as text (nothing is compiled or run): the dense
adjacency matrices of tests/include/test_utils.hpp and
include/sygraph/io/matrices.hpp, and the answers its tests assert.  Each entry
keeps the file:line it came from.  The committed kat.json is the
authoritative fixture; it is regenerated only by hand, from the repository
root, with the path of a SYgraph checkout:

    python tests/golden/make_golden.py /path/to/SYgraph
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

if __name__ == "__main__" and len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py /path/to/SYgraph")
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else None
OUT = Path(__file__).resolve().parent / "kat.json"


def read(rel: str) -> list[str]:
    return (REF / rel).read_text().splitlines()


def find_line(lines: list[str], pattern: str, start: int = 0) -> int:
    rx = re.compile(pattern)
    for i in range(start, len(lines)):
        if rx.search(lines[i]):
            return i
    raise LookupError(pattern)


def matrix_literal(rel: str, name: str) -> dict:
    """A `name = "n\\n" "row\\n" ...;` string literal -> {n, rows, where}."""
    lines = read(rel)
    i = find_line(lines, rf"\b{name}\s*=")
    chunks = []
    j = i
    while True:
        chunks += re.findall(r'"((?:[^"\\]|\\.)*)"', lines[j])
        if lines[j].rstrip().endswith(";"):
            break
        j += 1
    text = "".join(chunks).replace("\\n", "\n")
    toks = text.split()
    n = int(toks[0])
    rows = [[int(x) for x in toks[1 + r * n:1 + (r + 1) * n]] for r in range(n)]
    return {"n": n, "rows": rows, "where": f"{rel}:{i + 1}-{j + 1}"}


def int_list(s: str) -> list[int]:
    return [int(x) for x in re.findall(r"-?\d+", s)]


def braces_after(lines: list[str], pattern: str) -> tuple[list[int], int]:
    i = find_line(lines, pattern)
    m = re.search(pattern + r".*?\{([^}]*)\}", lines[i])
    return int_list(m.group(1)), i + 1


def main() -> None:
    kat = {"reference": "unisa-hpc/SYgraph", "matrices": {}, "cases": []}
    for name in ("line_5", "star_5", "triangle_3", "weighted_directed_5"):
        kat["matrices"][name] = matrix_literal("tests/include/test_utils.hpp", name)
    for name in ("symmetric_6nodes", "two_cc"):
        kat["matrices"][name] = matrix_literal("include/sygraph/io/matrices.hpp", name)

    cases = kat["cases"]

    # tests/operators/advance.cpp: BFS by advance from 0 on symmetric_6nodes
    f = "tests/operators/advance.cpp"
    vals, ln = braces_after(read(f), r"expected_distances")
    cases.append({"name": "advance_push_bfs_depths", "matrix": "symmetric_6nodes", "source": 0,
                  "load_balancers": ["workgroup_mapped", "bucketing"], "expected": vals, "where": f"{f}:{ln}"})

    # tests/operators/advance_graph.cpp: advance::vertices marks vertices with degree != 0
    f = "tests/operators/advance_graph.cpp"
    lines = read(f)
    i = find_line(lines, r"expected_visited")
    flags = [1 if t == "true" else 0 for t in re.findall(r"true|false", lines[i].split("{", 1)[1])]
    cases.append({"name": "advance_graph_nonzero_degree", "matrix": "two_cc", "expected": flags,
                  "where": f"{f}:{i + 1}"})

    # tests/operators/advance_pull.cpp: in = {0, 1}; vertex 2 activated; bucketing visits vertex 2 once
    f = "tests/operators/advance_pull.cpp"
    lines = read(f)
    ins = [int(x) for x in re.findall(r"in_frontier\.insert\((\d+)\)", "\n".join(lines))]
    a = find_line(lines, r"assert\(workgroup_default_active\[2\]\)")
    b = find_line(lines, r"assert\(bucketing_visits == 1\)")
    w = find_line(lines, r"assert\(workgroup_visits >= 1\)")
    cases.append({"name": "advance_pull_short_circuit", "matrix": "symmetric_6nodes", "in_frontier": ins,
                  "activated": [2], "bucketing_visits_of_2": 1, "workgroup_visits_of_2_at_least": 1,
                  "where": f"{f}:{a + 1},{w + 1},{b + 1}"})

    # tests/operators/filter_compute.cpp on star_5
    f = "tests/operators/filter_compute.cpp"
    lines = read(f)
    i = find_line(lines, r"for \(uint v : \{")
    inp = int_list(lines[i].split("{", 1)[1].split("}", 1)[0])
    e, le = braces_after(lines, r"expectFrontier\(output, std::vector<uint>")
    p, lp = braces_after(lines, r"expectFrontier\(input, std::vector<uint>")
    s, ls = braces_after(lines, r"expected_seen")
    r = find_line(lines, r"assert\(sum == ")
    total = int(re.search(r"sum == (\d+)", lines[r]).group(1))
    lt = int(re.search(r"vertex < (\d+)", lines[find_line(lines, r"filter::inplace")]).group(1))
    cases.append({"name": "filter_compute", "matrix": "star_5", "input": inp, "external_even": e,
                  "inplace_remove_less_than": lt, "after_inplace": p, "execute_seen": s, "reduce_sum": total,
                  "where": f"{f}:{le},{lp},{ls},{r + 1}"})

    # tests/operators/intersection.cpp on line_5
    f = "tests/operators/intersection.cpp"
    lines = read(f)
    i1 = find_line(lines, r"lhs\.insert")
    i2 = find_line(lines, r"rhs\.insert")
    x, lx = braces_after(lines, r"expectFrontier\(out, std::vector<uint>")
    cases.append({"name": "intersection", "matrix": "line_5",
                  "lhs": int_list(lines[i1].split("{", 1)[1].split("}", 1)[0]),
                  "rhs": int_list(lines[i2].split("{", 1)[1].split("}", 1)[0]), "expected": x, "where": f"{f}:{lx}"})

    # tests/frontier/mlb_frontier.cpp on star_5
    f = "tests/frontier/mlb_frontier.cpp"
    lines = read(f)
    ins = [int(v) for v in re.findall(r"frontier\.insert\((\d+)\)", "\n".join(lines))]
    rem = [int(v) for v in re.findall(r"frontier\.remove\((\d+)\)", "\n".join(lines))]
    exps = [int_list(m) for m in re.findall(r"expectFrontier\(frontier, std::vector<uint>\{([^}]*)\}", "\n".join(lines))]
    cases.append({"name": "mlb_frontier", "matrix": "star_5", "inserts": ins, "removes": rem,
                  "after_insert": exps[0], "after_remove": exps[1], "after_load": exps[2],
                  "where": f"{f}:{find_line(lines, 'expectFrontier') + 1}"})

    # tests/algorithms/bfs.cpp on line_5 from 0
    f = "tests/algorithms/bfs.cpp"
    lines = read(f)
    expd = [int_list(m) for m in re.findall(r"std::array<uint, 5>\{([^}]*)\}", "\n".join(lines))]
    it = int(re.search(r"iterations == (\d+)", "\n".join(lines)).group(1))
    cases.append({"name": "bfs_line5", "matrix": "line_5", "source": 0, "expected_push": expd[0],
                  "expected_pull": expd[1], "expected_hybrid": expd[2], "hybrid_alpha": 1.0, "hybrid_beta": 1.0,
                  "hybrid_iterations": it, "where": f"{f}:{find_line(lines, 'iterations ==') + 1}"})

    # tests/algorithms/sssp.cpp on weighted_directed_5 (directed, weighted) from 0
    f = "tests/algorithms/sssp.cpp"
    lines = read(f)
    d, ld = braces_after(lines, r"std::array<uint, 5>")
    cases.append({"name": "sssp_weighted_directed5", "matrix": "weighted_directed_5", "source": 0, "directed": True,
                  "expected": d, "where": f"{f}:{ld}"})

    # tests/algorithms/tc.cpp on triangle_3
    f = "tests/algorithms/tc.cpp"
    lines = read(f)
    i = find_line(lines, r"getNumTriangles\(\) == ")
    cases.append({"name": "tc_triangle3", "matrix": "triangle_3",
                  "expected": int(re.search(r"== (\d+)", lines[i]).group(1)), "where": f"{f}:{i + 1}"})

    # tests/algorithms/cc.cpp and bc.cpp run without assertions: record the inputs only
    cases.append({"name": "cc_two_cc_runs", "matrix": "two_cc", "sources": [0, 5], "asserts": False,
                  "where": "tests/algorithms/cc.cpp:3-16"})
    cases.append({"name": "bc_line5_runs", "matrix": "line_5", "source": 0, "asserts": False,
                  "where": "tests/algorithms/bc.cpp:3-11"})

    # binary CSR header constants (io/read_csr.hpp:22-24)
    lines = read("include/sygraph/io/read_csr.hpp")
    i = find_line(lines, r"magic = 0x")
    kat["binary_csr"] = {"magic": int(re.search(r"0x([0-9A-Fa-f]+)", lines[i]).group(1), 16),
                         "directed_mask": 1, "weighted_mask": 2, "where": f"include/sygraph/io/read_csr.hpp:{i + 1}"}

    OUT.write_text(json.dumps(kat, indent=1) + "\n")
    print(f"wrote {OUT} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
