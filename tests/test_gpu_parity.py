"""Parity of the CUDA engine with the reference (through the C ABI).

Costs must be bit-exact against the reference's own outputs (golden fixtures
made by the reference PrunedDP++ / D-PrunedDP++ binaries) and against the
oracle restatement on further seeded inputs; every returned tree must be a
tree of that weight touching every queried group, with hop diameter <= D for
the D- variants."""
import numpy as np
import pytest

import gst_b200
from gst_b200 import datagen as dg
import oracle

pytestmark = pytest.mark.gpu


def _load(engine, g, gr):
    engine.load_graph(g.rowptr, g.col, g.w)
    engine.load_groups(gr.ptr, gr.mem)


def _check_tree(g, gr, ids, r, D=-1):
    if not r.feasible:
        return
    code = oracle.validate(g, gr, ids, r.edges, r.root, r.cost, D)
    assert code == 0, (list(ids), D, r.cost, code)


@pytest.mark.parametrize("name", ["toy60", "s3000", "c1", "edge"])
def test_plain_matches_reference_goldens(engine, golden, name):
    fx, g, gr = golden(name)
    _load(engine, g, gr)
    for k, qs in fx["queries"].items():
        res = engine.solve_batch(qs)
        for ids, r, want in zip(qs, res, fx["reference"]["prunedpp"][k]):
            assert r.status == 0
            assert r.cost == want, (name, ids, r.cost, want)
            _check_tree(g, gr, ids, r)


@pytest.mark.parametrize("name", ["toy60", "s3000", "c1", "edge"])
def test_diameter_bound_matches_reference_goldens(engine, golden, name):
    fx, g, gr = golden(name)
    _load(engine, g, gr)
    for h in fx["reference"]["hop"]:
        qs = fx["queries"][str(h["k"])][: h["n"]]
        res = engine.solve_batch(qs, [h["D"]] * len(qs))
        for ids, r, want in zip(qs, res, h["costs"]):
            assert r.status == 0
            assert r.cost == want, (name, ids, h["D"], r.cost, want)
            _check_tree(g, gr, ids, r, h["D"])


def test_edge_cases(engine, golden):
    fx, g, gr = golden("edge")
    _load(engine, g, gr)
    # k = 1, infeasible (other component), empty group, duplicate ids
    for k, qs in fx["queries"].items():
        for ids, want in zip(qs, fx["reference"]["prunedpp"][k]):
            r = engine.solve(ids)
            assert r.cost == want, (ids, r.cost, want)
            assert r.feasible == (want < oracle.INF)
            if want == 0:
                assert len(r.edges) == 0 and r.root >= 0
    with pytest.raises(gst_b200.GstError) as e:
        engine.solve([0, 99])
    assert e.value.status == 1  # group id out of range
    with pytest.raises(gst_b200.GstError) as e:
        engine.solve([0, 1, 2], D=16)
    assert e.value.status == 6  # D above GST_MAX_D


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_graphs_against_unpruned_dpbf(engine, seed):
    g = dg.ba_graph(400 + 300 * seed, 2 + seed, 1, 30 * seed, seed=100 + seed, spanning_path=seed % 2 == 1)
    gr = dg.make_groups(g.V, 40, seed=200 + seed, uniform=(1, 8))
    _load(engine, g, gr)
    for k in (2, 3, 4, 5, 6, 7):
        qs = [q for q, _ in dg.make_queries(gr.n, 4, k, seed=300 + 10 * seed + k)]
        res = engine.solve_batch(qs)
        for ids, r in zip(qs, res):
            want = oracle.dpbf(g, gr, ids)[0]
            assert r.status == 0 and r.cost == want, (seed, list(ids), r.cost, want)
            _check_tree(g, gr, ids, r)


@pytest.mark.parametrize("seed", [4, 5])
def test_random_graphs_against_hop_oracle(engine, seed):
    g = dg.ba_graph(500, 3, 1, 40, seed=100 + seed)
    gr = dg.make_groups(g.V, 30, seed=200 + seed, uniform=(1, 5))
    _load(engine, g, gr)
    for k in (2, 3, 4, 5):
        qs = [q for q, _ in dg.make_queries(gr.n, 3, k, seed=400 + k)]
        for D in (0, 1, 2, 3, 5):
            res = engine.solve_batch(qs, [D] * len(qs))
            for ids, r in zip(qs, res):
                want = oracle.hop(g, gr, ids, D)[0]
                assert r.status == 0 and r.cost == want, (list(ids), D, r.cost, want)
                _check_tree(g, gr, ids, r, D)


def test_cost_monotone_in_D_and_plain_limit(engine, golden):
    fx, g, gr = golden("toy60")
    _load(engine, g, gr)
    for ids in fx["queries"]["3"][:6]:
        plain = engine.solve(ids).cost
        costs = [engine.solve(ids, D=D).cost for D in range(0, 16)]
        assert all(a >= b for a, b in zip(costs, costs[1:]))
        assert costs[-1] == plain  # 15 hops exceed this graph's tree depths


def test_query_permutation_invariance(engine, golden):
    fx, g, gr = golden("s3000")
    _load(engine, g, gr)
    rng = np.random.default_rng(5)
    qs = fx["queries"]["5"][:6]
    perm = [list(rng.permutation(q)) for q in qs]
    a = engine.solve_batch(qs)
    b = engine.solve_batch(perm)
    assert [r.cost for r in a] == [r.cost for r in b]


def test_batch_equals_one_at_a_time(engine, golden):
    fx, g, gr = golden("s3000")
    _load(engine, g, gr)
    qs = fx["queries"]["5"] + fx["queries"]["7"]
    Ds = [-1, 2, 3, -1, 4, -1] * 3
    batch = engine.solve_batch(qs, Ds[: len(qs)])
    for ids, D, r in zip(qs, Ds, batch):
        alone = engine.solve(ids, D=D)
        assert alone.cost == r.cost


def test_round_limit_surfaces_as_status(golden):
    """A forced tiny device round budget must fail the query with
    GST_E_LIMIT and leave the engine usable (fault injected on the host)."""
    fx, g, gr = golden("s3000")
    e = gst_b200.Engine(device=0, arena_bytes=1 << 30, max_rounds=3)
    _load(e, g, gr)
    r = e.solve(fx["queries"]["5"][0])
    assert r.status == 7
    e.close()
    e2 = gst_b200.Engine(device=0, arena_bytes=1 << 30, max_rounds=100000)
    _load(e2, g, gr)
    assert e2.solve(fx["queries"]["5"][0]).cost == fx["reference"]["prunedpp"]["5"][0]
    e2.close()


def test_unsupported_and_oversized_requests(golden):
    fx, g, gr = golden("c1")
    e = gst_b200.Engine(device=0, arena_bytes=64 << 20, max_rounds=100000)
    _load(e, g, gr)
    with pytest.raises(gst_b200.GstError) as err:
        e.solve(list(range(8)))
    assert err.value.status == 6  # k above GST_MAX_K
    # a k=7, D=15 table of 10k vertices needs ~82 MB: more than the whole arena
    r = e.solve(list(range(7)), D=15)
    assert r.status == 5  # GST_E_NOMEM, rejected at admission
    assert e.solve(fx["queries"]["3"][0]).cost == fx["reference"]["prunedpp"]["3"][0]
    e.close()
