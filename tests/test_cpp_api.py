"""The C++ header API as a drop-in: tests/cpp/api_kat.cu restates the
reference's own test programs against include/sygraph/ (device lambdas,
templated advances) and must print ALL OK on the GPU."""
import importlib.util
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _build_module():
    spec = importlib.util.spec_from_file_location("sg_build", ROOT / "sygraph_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_cpp_api_known_answers(golden):
    b = _build_module()
    b.build_library()
    exes = {p.name: p for p in b.build_cpp_tests()}
    exe = exes["api_kat"]
    args = []
    for name, m in golden["matrices"].items():
        args.append(f"{name}=" + ";".join([str(m["n"])] + [" ".join(map(str, r)) for r in m["rows"]]))
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stderr
    assert "ALL OK" in r.stdout
