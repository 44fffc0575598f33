"""The oracle restatement against the reference's own outputs (CPU only).

The fixtures hold what the reference PrunedDP++ / D-PrunedDP++ binaries
printed on seeded inputs (tests/golden/make_golden.py); the oracle must
reproduce every cost, and its trees must validate.  The unpruned exact DPBF
must agree too, which shows the reference's pruning kept the optimum."""
import numpy as np
import pytest

import oracle


@pytest.mark.parametrize("name", ["toy60", "s3000", "c1", "edge"])
def test_prunedpp_restatement_matches_reference(golden, name):
    fx, g, gr = golden(name)
    for k, qs in fx["queries"].items():
        want = fx["reference"]["prunedpp"][k]
        assert len(want) == len(qs)
        for ids, w in zip(qs, want):
            cost, edges, root, _ = oracle.prunedpp(g, gr, ids)
            assert cost == w, (name, ids, cost, w)
            if cost < oracle.INF:
                assert oracle.validate(g, gr, ids, edges, root, cost) == 0


@pytest.mark.parametrize("name", ["toy60", "s3000", "edge"])
def test_unpruned_dpbf_matches_reference(golden, name):
    fx, g, gr = golden(name)
    for k, qs in fx["queries"].items():
        for ids, w in zip(qs, fx["reference"]["prunedpp"][k]):
            cost, edges, root, _ = oracle.dpbf(g, gr, ids)
            assert cost == w, (name, ids, cost, w)
            if cost < oracle.INF:
                assert oracle.validate(g, gr, ids, edges, root, cost) == 0


@pytest.mark.parametrize("name", ["toy60", "s3000", "c1", "edge"])
def test_hop_restatement_matches_reference(golden, name):
    fx, g, gr = golden(name)
    for h in fx["reference"]["hop"]:
        qs = fx["queries"][str(h["k"])][: h["n"]]
        for ids, w in zip(qs, h["costs"]):
            cost, edges, root, _ = oracle.hop(g, gr, ids, h["D"])
            assert cost == w, (name, ids, h["D"], cost, w)


@pytest.mark.parametrize("name", ["toy60", "s3000", "c1", "edge"])
def test_lean_hop_restatement_matches_reference(golden, name):
    """The 4-bytes-per-state HOP restatement (which pins the C4 cells whose
    reference table does not fit) gives the reference's cost on every cell,
    and its rebuilt tree keeps the hop bound."""
    fx, g, gr = golden(name)
    for h in fx["reference"]["hop"]:
        qs = fx["queries"][str(h["k"])][: h["n"]]
        for ids, w in zip(qs, h["costs"]):
            cost, edges, root, _ = oracle.hop_lean(g, gr, ids, h["D"])
            assert cost == w, (name, ids, h["D"], cost, w)
            if cost < oracle.INF:
                assert oracle.validate(g, gr, ids, edges, root, cost, h["D"]) == 0


def test_hop_properties_on_oracle(golden):
    """Cost is non-increasing in D and reaches the plain optimum for large D."""
    fx, g, gr = golden("toy60")
    for ids in fx["queries"]["3"][:8]:
        plain = oracle.dpbf(g, gr, ids)[0]
        prev = None
        for D in range(0, 8):
            c = oracle.hop(g, gr, ids, D)[0]
            if prev is not None:
                assert c <= prev
            prev = c
        assert oracle.hop(g, gr, ids, 59)[0] == plain


def test_validator_rejects_bad_trees(golden):
    fx, g, gr = golden("toy60")
    ids = fx["queries"]["3"][0]
    cost, edges, root, _ = oracle.prunedpp(g, gr, ids)
    assert oracle.validate(g, gr, ids, edges, root, cost) == 0
    assert oracle.validate(g, gr, ids, edges, root, cost + 1) == 4       # wrong weight
    if len(edges) > 1:
        assert oracle.validate(g, gr, ids, edges[1:], root, cost) != 0   # cover/connectivity
    bad = edges.copy()
    bad[0, 2] += 1
    assert oracle.validate(g, gr, ids, bad, root, cost) == 1              # weight mismatch


def test_c2_fixture_regenerates_and_pins_the_restatement(golden):
    """The full-size C2 fixture: the generator reproduces the benchmark graph
    (checksum), and the restatement equals the reference on its first two
    plain queries (a few seconds each; the GPU test covers all of them)."""
    fx, g, gr = golden("c2")
    qs, want = fx["queries"]["5"], fx["reference"]["prunedpp"]["5"]
    for ids, w in zip(qs[:2], want[:2]):
        assert oracle.prunedpp(g, gr, ids)[0] == w


@pytest.mark.parametrize("name", ["c3", "c4", "c2_batch"])
def test_benchmark_size_fixtures_reproduce(name):
    """The C3 / C4 / C2-batch fixtures (made by tests/golden/make_golden_large.py from the
    reference binaries) still describe what the generator builds, and their
    queries are the workload's own queries at the recorded indices."""
    import json
    import os
    import sys
    from gst_b200 import datagen as dg
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    import make_golden as mg
    with open(os.path.join(here, f"{name}.json")) as f:
        fx = json.load(f)
    wl = {"c4": dg.config_c4, "c3": dg.config_c3, "c2_batch": dg.config_c2}[name](1, n_queries=300)
    assert mg.checksum(wl.graph, wl.groups) == fx["checksum"]
    pinned = 0
    for c in fx["cells"]:
        if not c.get("costs"):
            assert c.get("not_pinned")
            continue
        # who printed the costs: a reference binary, or (only for a cell the
        # reference cannot run, with the reason recorded) the restatement
        assert c["program"] in ("PrunedDP++", "D-PrunedDP++", "oracle.hop_lean")
        if c["program"] == "oracle.hop_lean":
            assert c["D"] >= 0 and c.get("reference_not_run")
        for i, q, cost in zip(c["idx"], c["queries"], c["costs"]):
            ids, D = wl.queries[i]
            assert ids.tolist() == q and D == c["D"] and len(q) == c["k"]
            assert cost == oracle.INF or 0 < cost < oracle.INF
            pinned += 1
    assert pinned >= {"c4": 130, "c3": 18, "c2_batch": 300}[name]
