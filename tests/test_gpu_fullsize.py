"""Parity at the benchmark sizes (C2: 170k vertices, k=5; a C3-shaped
diameter-bounded k=7 case) through size-independent properties, plus a sample
against the oracle restatement where it finishes in seconds.

* every returned tree is a tree of exactly the reported weight touching every
  group (and of hop diameter <= D for the D- variants);
* the batch and the one-query-per-call forms agree;
* permuting a query's group ids does not change the cost;
* costs are non-increasing in D and never below the plain optimum;
* on C2, a sample of queries equals the PrunedDP++ restatement."""
import numpy as np
import pytest

import gst_b200
from gst_b200 import datagen as dg
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2():
    wl = dg.config_c2(1, n_queries=24)
    e = gst_b200.Engine(device=0, arena_bytes=8 << 30, max_rounds=500000)
    e.load_graph(wl.graph.rowptr, wl.graph.col, wl.graph.w)
    e.load_groups(wl.groups.ptr, wl.groups.mem)
    yield wl, e
    e.close()


def test_c2_trees_batch_single_permutation(c2):
    wl, e = c2
    qs = [q for q, _ in wl.queries]
    batch = e.solve_batch(qs)
    rng = np.random.default_rng(11)
    for i, (q, r) in enumerate(zip(qs, batch)):
        assert r.status == 0 and r.feasible
        assert oracle.validate(wl.graph, wl.groups, q, r.edges, r.root, r.cost) == 0
        if i < 6:
            assert e.solve(q).cost == r.cost
            assert e.solve(rng.permutation(q)).cost == r.cost


def test_c2_sample_equals_prunedpp_restatement(c2):
    wl, e = c2
    for q, _ in wl.queries[:2]:
        want = oracle.prunedpp(wl.graph, wl.groups, q)[0]
        assert e.solve(q).cost == want


def test_c2_diameter_bound_properties(c2):
    wl, e = c2
    for q, _ in wl.queries[:4]:
        plain = e.solve(q).cost
        prev = None
        for D in (2, 3, 4, 5, 8):
            r = e.solve(q, D)
            if r.feasible:
                assert oracle.validate(wl.graph, wl.groups, q, r.edges, r.root, r.cost, D) == 0
                assert r.cost >= plain
            if prev is not None:
                assert r.cost <= prev
            prev = r.cost


def test_c3_shaped_k7_diameter_bound():
    """1M-vertex BA graph (m=10, w U[1,1000]), k=7, D in {2..5}: trees valid,
    costs non-increasing in D, batch equals single."""
    g = dg.ba_graph(1_000_000, 10, 1, 1000, seed=1)
    gr = dg.make_groups(g.V, 10_000, seed=101, geometric=(10, 2, 500))
    qs = [q for q, _ in dg.make_queries(gr.n, 3, 7, seed=201)]
    e = gst_b200.Engine(device=0, arena_bytes=48 << 30, max_rounds=500000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    for q in qs:
        costs = []
        for D in (2, 3, 4, 5):
            r = e.solve(q, D)
            assert r.status == 0
            if r.feasible:
                assert oracle.validate(g, gr, q, r.edges, r.root, r.cost, D) == 0
            costs.append(r.cost)
        assert all(a >= b for a, b in zip(costs, costs[1:]))
    batch = e.solve_batch(qs, [3, 4, 5])
    for q, D, r in zip(qs, [3, 4, 5], batch):
        assert r.cost == e.solve(q, D).cost
    e.close()


def test_c2_equals_the_reference_binaries(golden):
    """The C2 benchmark graph and groups, 12 plain queries and 6 D-queries
    (D = 4, 5): costs equal what the reference PrunedDP++ / D-PrunedDP++
    printed (tests/golden/c2.json), batched and one per call."""
    fx, g, gr = golden("c2")
    e = gst_b200.Engine(device=0, arena_bytes=8 << 30, max_rounds=500000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    qs = fx["queries"]["5"]
    got = [r.cost for r in e.solve_batch(qs)]
    assert got == fx["reference"]["prunedpp"]["5"]
    assert e.solve(qs[0]).cost == got[0]
    for h in fx["reference"]["hop"]:
        batch = e.solve_batch(qs[: h["n"]], [h["D"]] * h["n"])
        assert [r.cost for r in batch] == h["costs"], h["D"]
        for q, r in zip(qs, batch):
            if r.feasible:
                assert oracle.validate(g, gr, q, r.edges, r.root, r.cost, h["D"]) == 0
    e.close()


def _large_fixture(name):
    """A reference-pinned fixture at benchmark size (tests/golden/<name>.json,
    made by tests/golden/make_golden_large.py) and its regenerated inputs."""
    import json
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    path = os.path.join(here, f"{name}.json")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated")
    with open(path) as f:
        fx = json.load(f)
    sys.path.insert(0, here)
    import make_golden as mg
    wl = {"c4": dg.config_c4, "c3": dg.config_c3, "c2_batch": dg.config_c2}[name](1, n_queries=300)
    assert mg.checksum(wl.graph, wl.groups) == fx["checksum"], f"{name}: generator no longer reproduces the fixture"
    cells = [c for c in fx["cells"] if c.get("costs") and all(x is not None for x in c["costs"])]
    if not cells:
        pytest.skip(f"{path} has no finished cell yet")
    return fx, wl, cells


@pytest.mark.parametrize("name", ["c4", "c3", "c2_batch"])
def test_benchmark_size_costs_equal_the_reference_binaries(name):
    """C4 (4M vertices, the headline workload), C3 (1M vertices, k=7 with
    D in {2..5}) and the whole 300-query C2 batch (170k vertices, k=5): every
    pinned query of every (k, D) cell equals the cost the
    reference PrunedDP++ / D-PrunedDP++ printed (for C4's k=7 D-bounded cells,
    whose reference table does not fit in memory, the cost of the HOP_cpu
    restatement oracle.hop_lean), solved as one batch; the first query of each
    cell also one per call; every tree passes the checker."""
    fx, wl, cells = _large_fixture(name)
    e = gst_b200.Engine(device=0, max_rounds=2000000)
    e.load_graph(wl.graph.rowptr, wl.graph.col, wl.graph.w)
    e.load_groups(wl.groups.ptr, wl.groups.mem)
    qs, Ds, want = [], [], []
    for c in cells:
        for q, cost in zip(c["queries"], c["costs"]):
            qs.append(q)
            Ds.append(c["D"])
            want.append(cost)
    got = e.solve_batch(qs, Ds)
    assert [r.cost for r in got] == want
    for q, D, r in zip(qs, Ds, got):
        assert r.status == 0
        if r.feasible:
            assert oracle.validate(wl.graph, wl.groups, q, r.edges, r.root, r.cost, D) == 0
    for c in cells:
        assert e.solve(c["queries"][0], c["D"]).cost == c["costs"][0], (c["k"], c["D"])
    e.close()
