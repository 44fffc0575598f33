import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu4gst-1_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    """Regenerates a golden dataset from its recipe and checks the checksum."""
    from gst_b200 import datagen as dg
    sys.path.insert(0, GOLDEN)
    import make_golden as mg

    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        fx = json.load(f)
    if name == "edge":
        g = dg.Graph(np.array(fx["graph"]["rowptr"], np.int64), np.array(fx["graph"]["col"], np.int32),
                     np.array(fx["graph"]["w"], np.int32))
        gr = dg.Groups(np.array(fx["groups"]["ptr"], np.int64), np.array(fx["groups"]["mem"], np.int32))
    else:
        g, gr, _ = mg.build(fx["spec"])
    assert mg.checksum(g, gr) == fx["checksum"], f"{name}: generator no longer reproduces the fixture"
    return fx, g, gr


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = load_golden(name)
        return cache[name]
    return get


@pytest.fixture(scope="session")
def engine():
    import gst_b200
    e = gst_b200.Engine(device=0, arena_bytes=4 << 30, max_rounds=200000)
    yield e
    e.close()
