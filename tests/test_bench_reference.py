"""The CPU reference arm of bench.py keeps the bench's JSON contract: one
line with the headline metric, impl "reference", a cpu_baseline describing
the run and an e2e object without host-device copies.  It runs the GPU arm's
workload (same config object) and loads nothing of sygraph_b200."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


RUNNER = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED_PRODUCT", "libsygraph_b200" in maps or "sygraph_b200" in sys.modules)
"""


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "-c", RUNNER], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    assert "LOADED_PRODUCT False" in r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "GTEPS" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    sys.path.insert(0, str(ROOT))
    import bench
    assert d["config"] == bench.bench_config(1 << bench.SCALE, d["config"]["m"])
    assert d["config"]["sources_per_step"] == 64 and d["config"]["m"] == 128301086


def test_every_traffic_key_of_the_bench_has_a_capture():
    """Each kernel whose `traffic` the bench line reports has its ncu DRAM
    bytes in profiles/traffic.json and a summary in profiles/ naming the
    profiling case that captured it."""
    import re

    src = (ROOT / "bench.py").read_text()
    keys = set(re.findall(r'ncu_traffic\("([a-z_0-9]+)"\)', src))
    traffic = json.loads((ROOT / "profiles" / "traffic.json").read_text())
    assert keys and keys <= set(traffic), keys - set(traffic)
    assert all(isinstance(traffic[k], int) and traffic[k] > 0 for k in keys)
    summaries = " ".join(p.read_text() for p in (ROOT / "profiles").glob("*.md"))
    cases = set(re.search(r'"--profile", choices=\[([^\]]*)\]', src).group(1).replace('"', "").replace(" ", "").split(","))
    for case in cases:
        assert f"--profile {case}" in summaries, case
