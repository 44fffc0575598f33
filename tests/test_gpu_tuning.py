"""Launch and scheduling parameters change speed, never a cost: the same
mixed batch (plain and D-bounded queries, k = 3..5) solved under every grow
lane count, both merge/grow schedules (in sequence and on two streams),
small chunks, wide cost buckets and few slots gives the default's costs and
valid trees; out-of-range parameters are refused."""
import pytest

import gst_b200
from gst_b200 import datagen as dg
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    g = dg.ba_graph(20000, 4, 1, 100, seed=41, spanning_path=True)
    gr = dg.make_groups(g.V, 400, seed=42, geometric=(8, 2, 100))
    qs = dg.make_queries(gr.n, 24, [3, 4, 5], seed=43, D=lambda r: -1 if r.random() < 0.5 else int(r.integers(2, 5)))
    e = gst_b200.Engine(device=0, arena_bytes=2 << 30, max_rounds=500000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    want = [r.cost for r in e.solve_batch([q for q, _ in qs], [D for _, D in qs])]
    yield g, gr, qs, e, want
    e.close()


@pytest.mark.parametrize("tuning", [
    {"grow_lanes": 8}, {"grow_lanes": 32}, {"overlap": 2},
    {"overlap": 2, "grow_lanes": 32, "rounds_per_poll": 4},
    {"chunk_pairs": [[256, 256]] * 8, "bucket_mult": [4] * 8},
    {"max_slots": 5, "rounds_per_poll": 16},
])
def test_tuning_keeps_every_cost(setup, tuning):
    g, gr, qs, e, want = setup
    default = e.get_tuning()
    e.set_tuning(tuning)
    try:
        got = e.solve_batch([q for q, _ in qs], [D for _, D in qs])
        assert [r.cost for r in got] == want
        for (q, D), r in zip(qs, got):
            assert r.status == 0
            if r.feasible:
                assert oracle.validate(g, gr, q, r.edges, r.root, r.cost, D) == 0
    finally:
        e.set_tuning({"grow_lanes": default["grow_lanes"], "overlap": default["overlap"],
                      "rounds_per_poll": default["rounds_per_poll"], "max_slots": default["max_slots"],
                      "chunk_pairs": default["chunk_pairs"], "bucket_mult": default["bucket_mult"]})


def test_tuning_rejects_out_of_range(setup):
    e = setup[3]
    for bad in ({"grow_lanes": 12}, {"overlap": 3}, {"max_slots": 5000}):
        with pytest.raises(gst_b200.GstError):
            e.set_tuning(bad)
