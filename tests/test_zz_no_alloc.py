"""gst_solve_noalloc: the allocation-free entry point.

It exists for callers that cannot allocate memory once they are running (a
process that reserved all device memory up front, code in allocation-free
sections, plugin hosts that forbid cudaMalloc after start-up).  Such a caller
owns the graph and groups in device memory and passes pointers to them; all
scratch comes from a static device array of the library.  Through the C ABI,
its cost and root must equal the regular gst_solve entry point's, exactly as
every other cost in these tests, on two calls in a row (the shared scratch
keeps the previous call's contents, so each call must re-initialise it).
This file is collected last so that a failing run has already run the rest."""
import ctypes

import numpy as np
import pytest

import gst_b200

pytestmark = pytest.mark.gpu


def _device_inputs(torch, g, gr):
    adj = np.empty((g.E, 2), np.int32)
    adj[:, 0] = g.col
    adj[:, 1] = g.w
    return {
        "rowptr": torch.from_numpy(np.ascontiguousarray(g.rowptr)).cuda(),
        "adj": torch.from_numpy(adj.reshape(-1)).cuda(),
        "gptr": torch.from_numpy(np.ascontiguousarray(gr.ptr)).cuda(),
        "gmem": torch.from_numpy(np.ascontiguousarray(gr.mem)).cuda(),
    }


def _noalloc(lib, g, gr, dev, ids, D):
    q = np.ascontiguousarray(ids, np.int32)
    cost = ctypes.c_int64(-1)
    root = ctypes.c_int32(-2)
    st = lib.gst_solve_noalloc(g.V, g.E, dev["rowptr"].data_ptr(), dev["adj"].data_ptr(), gr.n,
                               dev["gptr"].data_ptr(), dev["gmem"].data_ptr(), q.ctypes.data, len(q), int(D),
                               None, ctypes.byref(cost), ctypes.byref(root))
    return st, cost.value, root.value


@pytest.mark.parametrize("name", ["s3000", "c1"])
def test_noalloc_equals_solve_on_two_calls_in_a_row(golden, name):
    import torch
    fx, g, gr = golden(name)
    lib = gst_b200.load_library()
    dev = _device_inputs(torch, g, gr)
    torch.cuda.synchronize()
    e = gst_b200.Engine(device=0, arena_bytes=1 << 30, max_rounds=200000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    cases = []
    for k, qs in fx["queries"].items():
        for ids in qs[:3]:
            cases += [(ids, -1), (ids, 3)]
        cases.append((qs[0], 0))  # D = 0: one label, its own sizing path
    for ids, D in cases:
        want = e.solve(ids, D)
        for _ in range(2):
            st, cost, root = _noalloc(lib, g, gr, dev, ids, D)
            assert st == 0, gst_b200.load_library().gst_last_error()
            assert cost == want.cost, (ids, D, cost, want.cost)
            assert root == (want.root if want.feasible else -1)
    e.close()


def test_noalloc_rejects_queries_beyond_its_scratch(golden):
    import torch
    fx, g, gr = golden("c1")
    lib = gst_b200.load_library()
    dev = _device_inputs(torch, g, gr)
    torch.cuda.synchronize()
    # k = 7 with D = 15 on 10,000 vertices needs about 82 MiB of table alone
    st, cost, root = _noalloc(lib, g, gr, dev, list(range(7)), 15)
    assert st == 5  # GST_E_NOMEM
    assert b"static maximum" in lib.gst_last_error()


def test_noalloc_wide_weights_and_no_device_allocation():
    """Weights U[1,1000] on a 20,000-vertex graph (the bucket width comes from
    the graph, as in the engine), compared with gst_solve; after a warm-up
    call, further calls leave the device's free memory unchanged: the entry
    point allocates nothing, and nothing it loads grows later."""
    import torch
    from gst_b200 import datagen as dg
    g = dg.ba_graph(20000, 4, 1, 1000, seed=31, spanning_path=True)
    gr = dg.make_groups(g.V, 300, seed=32, geometric=(8, 2, 100))
    qs = [q for q, _ in dg.make_queries(gr.n, 6, [3, 4, 5], seed=33)]
    lib = gst_b200.load_library()
    dev = _device_inputs(torch, g, gr)
    torch.cuda.synchronize()
    e = gst_b200.Engine(device=0, arena_bytes=1 << 30, max_rounds=200000)
    e.load_graph(g.rowptr, g.col, g.w)
    e.load_groups(gr.ptr, gr.mem)
    cases = [(q, D) for q in qs for D in (-1, 2)]
    want = [e.solve(q, D) for q, D in cases]
    e.close()
    torch.cuda.synchronize()
    st, _, _ = _noalloc(lib, g, gr, dev, cases[0][0], cases[0][1])  # warm-up
    assert st == 0, lib.gst_last_error()
    free0, _ = torch.cuda.mem_get_info()
    for (q, D), w in zip(cases, want):
        st, cost, root = _noalloc(lib, g, gr, dev, q, D)
        assert st == 0, lib.gst_last_error()
        assert cost == w.cost, (list(q), D, cost, w.cost)
        assert root == (w.root if w.feasible else -1)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
