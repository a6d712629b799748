import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger graphs")


def _gpu_present() -> bool:
    try:
        import sygraph_b200 as sg
    except ImportError:
        return False
    return sg.device_count() > 0


def pytest_collection_modifyitems(config, items):
    if any(it.get_closest_marker("gpu") for it in items):
        if not _gpu_present():
            skip = pytest.mark.skip(reason="no CUDA device in this process")
            for it in items:
                if it.get_closest_marker("gpu"):
                    it.add_marker(skip)


@pytest.fixture(scope="session")
def sg():
    import sygraph_b200
    return sygraph_b200


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


@pytest.fixture(scope="session")
def golden():
    import json
    return json.loads((ROOT / "tests" / "golden" / "kat.json").read_text())


_GRAPH_CACHE = {}


@pytest.fixture(scope="session")
def rmat(sg):
    """rmat(scale, **kw) -> CSR, cached per session."""

    def make(scale, **kw):
        key = (scale, tuple(sorted(kw.items())))
        if key not in _GRAPH_CACHE:
            _GRAPH_CACHE[key] = sg.io.rmat(scale, **kw)
        return _GRAPH_CACHE[key]

    return make
