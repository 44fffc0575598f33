"""Serving: continuous batching through the server API.

Requests submitted from several threads while others are on the GPU are
admitted as slots free up (a small slot count forces queueing); every
result must equal the same query solved alone."""
import threading
import time

import numpy as np
import pytest

import gst_b200
import oracle

pytestmark = pytest.mark.gpu


def test_results_in_the_mix_equal_results_alone(golden):
    fx, g, gr = golden("s3000")
    e = gst_b200.Engine(device=0, arena_bytes=2 << 30, max_slots=4, rounds_per_poll=2, max_rounds=200000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    qs = fx["queries"]["5"] + fx["queries"]["7"]
    Ds = [(-1 if i % 3 == 0 else 2 + i % 4) for i in range(len(qs))]
    alone = [e.solve(q, D) for q, D in zip(qs, Ds)]
    tickets = [None] * len(qs)
    rng = np.random.default_rng(3)
    delays = rng.exponential(0.002, size=len(qs))
    with e.server() as srv:
        def client(idx):
            for i in idx:
                time.sleep(delays[i])
                tickets[i] = srv.submit(qs[i], Ds[i])
        ths = [threading.Thread(target=client, args=(list(range(j, len(qs), 3)),)) for j in range(3)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        mixed = [srv.wait(t) for t in tickets]
        with pytest.raises(gst_b200.GstError) as err:
            srv.wait(tickets[0])  # a result is handed out once
        assert err.value.status == 8
    for q, D, a, m in zip(qs, Ds, alone, mixed):
        assert m.status == 0
        assert m.cost == a.cost, (q, D, m.cost, a.cost)
        if m.feasible:
            assert oracle.validate(g, gr, q, m.edges, m.root, m.cost, D) == 0
    # the engine serves batch calls again once the server stopped
    assert e.solve(qs[0], Ds[0]).cost == alone[0].cost
    e.close()


def test_server_rejects_batch_calls_while_running(golden):
    fx, g, gr = golden("toy60")
    e = gst_b200.Engine(device=0, arena_bytes=256 << 20, max_rounds=100000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    srv = e.server()
    try:
        with pytest.raises(gst_b200.GstError) as err:
            e.solve(fx["queries"]["3"][0])
        assert err.value.status == 8  # GST_E_STATE
        t = srv.submit(fx["queries"]["3"][0])
        assert srv.wait(t, timeout_ms=60000).cost == fx["reference"]["prunedpp"]["3"][0]
    finally:
        srv.stop()
    e.close()
