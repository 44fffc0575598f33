"""Host-side pieces of the benchmark and the autotuner that need no GPU: the
fixture parity check raises on a single differing cost, the class weighting
of the one-query-per-call sample, and the tuning file round trip."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from gst_b200 import autotune  # noqa: E402


@pytest.fixture(scope="module")
def c4():
    return bench.make_workload("c4", 0)


def test_fixture_parity_accepts_the_reference_costs_and_rejects_one_change(c4):
    with open(os.path.join(ROOT, "tests", "golden", "c4.json")) as f:
        fx = json.load(f)
    costs = [None] * len(c4.queries)
    for c in fx["cells"]:
        for i, want in zip(c["idx"], c["costs"] or []):
            costs[i] = want
    got = bench.fixture_parity("c4", c4, costs)
    assert got["equal"] and got["queries_checked"] == sum(x is not None for x in costs)
    assert sum(got["by_program"].values()) == got["queries_checked"]
    i = next(i for i, x in enumerate(costs) if x is not None and x < 100000)
    costs[i] += 1  # a mistake planted in the checked values, on the CPU
    with pytest.raises(AssertionError):
        bench.fixture_parity("c4", c4, costs)


def test_query_classes_and_cpu_mix(c4):
    classes = {}
    for q, D in c4.queries:
        classes[bench.query_class(q, D)] = classes.get(bench.query_class(q, D), 0) + 1
    assert set(classes) == {"k3_plain", "k3_D", "k5_plain", "k5_D", "k7_plain", "k7_D"}
    assert sum(classes.values()) == 300
    # cores / the plain mix's mean time: 52 k=3, 51 k=5, 60 k=7 plain queries
    per_k = {3: 1.0, 5: 2.0, 7: 4.0}
    plain = [len(q) for q, D in c4.queries if D < 0]
    want = 16 / (sum(per_k[k] for k in plain) / len(plain))
    assert bench.cpu_mix_qps(per_k, c4.queries, 16) == pytest.approx(want)


def test_tuning_file_round_trip(tmp_path):
    tun = {"grow_lanes": 8, "rounds_per_poll": 8, "max_slots": 512, "overlap": 2,
           "chunk_pairs": [[1024, 1024]] * 8, "bucket_mult": [1] * 8}
    p = tmp_path / "t.json"
    autotune.save(str(p), {"tuning": tun, "final_median_ms": 1.0, "trace": []}, "c4")
    assert autotune.load(str(p)) == tun
    for w in ("c2", "c4"):
        committed = autotune.load(os.path.join(ROOT, "gpu4gst-1_b200", "tuning", f"{w}.json"))
        assert committed["grow_lanes"] in (8, 16, 32) and committed.get("overlap", 1) in (1, 2)
        assert len(committed["chunk_pairs"]) == 8 and len(committed["bucket_mult"]) == 8


def test_cpu_sample_positions_spread_over_the_class():
    assert bench.sample_positions(52, 3) == [0, 17, 34]
    assert bench.sample_positions(60, 3) == [0, 20, 40]
    assert bench.sample_positions(2, 3) == [0, 1]  # a class smaller than the sample
    assert bench.sample_positions(60, 1) == [0]
