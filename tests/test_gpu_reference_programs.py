"""The reference's own GPU programs against this engine, on the same inputs.

TrimCDP (plain, code/TrimCDP/src/DPQ.cu:558-575) and D-TrimCDP (diameter
bound, code/D-TrimCDP/src/DPQ.cu:229-242: the minimum over depth labels
d <= D of the full set) are built for sm_100a from the reference sources
into oracle/_ref/ by oracle/Makefile and run here with their own argv and
file formats.  Costs must be equal query by query, except where the
reference program is known to report something else: TrimCDP prints 0 for
an infeasible query (the CPU programs and this engine print 100000).  Each
such case is collected as a reference disagreement and must be one of the
known kinds; nothing else may differ.  The CPU reference (PrunedDP++ /
D-PrunedDP++) stays the authority: its costs are in the fixtures, and the
engine equals them in the other tests."""
import os
import tempfile

import numpy as np
import pytest

import gst_b200
from gst_b200 import datagen as dg
import oracle

pytestmark = pytest.mark.gpu


def _need(name):
    exe = oracle.ref_binary(name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (make -C oracle ref REF=<reference checkout>)")


def _run(name, g, gr, queries, k, D=None):
    d = tempfile.mkdtemp(prefix="gstrefgpu_")
    dg.write_dataset(d, "data", dg.Workload(g, gr, []), binary=False)
    dg.write_queries(os.path.join(d, f"data{k}.csv"), [(np.asarray(q), -1) for q in queries])
    rows = oracle.run_reference(name, d, "data", k, 0, len(queries) - 1, D=D, timeout=900)
    return [r[3] for r in rows]


def _compare(ref, ours):
    """Query indices where the reference program differs, by kind; raises on
    a difference of no known kind."""
    known = {"infeasible_reported_as_0": []}
    for i, (a, b) in enumerate(zip(ref, ours)):
        if a == b:
            continue
        if a == 0 and b == oracle.INF:
            known["infeasible_reported_as_0"].append(i)
        else:
            raise AssertionError(f"query {i}: reference GPU program {a}, engine {b}")
    return known


def test_trimcdp_equals_engine_on_c1_and_c2(golden):
    _need("TrimCDP")
    e = gst_b200.Engine(device=0, arena_bytes=4 << 30, max_rounds=500000)
    for name, n in (("c1", 50), ("c2", 6)):
        fx, g, gr = golden(name)
        k = 3 if name == "c1" else 5
        qs = fx["queries"][str(k)][:n]
        e.load_graph(g.rowptr, g.col, g.w)
        e.load_groups(gr.ptr, gr.mem)
        ours = [r.cost for r in e.solve_batch(qs)]
        assert ours == fx["reference"]["prunedpp"][str(k)][:n]
        ref = _run("TrimCDP", g, gr, qs, k)
        assert len(ref) == len(qs)
        _compare(ref, ours)
    e.close()


def test_d_trimcdp_equals_engine_on_c1_and_c2(golden):
    _need("D-TrimCDP")
    e = gst_b200.Engine(device=0, arena_bytes=4 << 30, max_rounds=500000)
    for name, k, D, n in (("c1", 3, 3, 20), ("c1", 3, 2, 10), ("c2", 5, 4, 3)):
        fx, g, gr = golden(name)
        qs = fx["queries"][str(k)][:n]
        e.load_graph(g.rowptr, g.col, g.w)
        e.load_groups(gr.ptr, gr.mem)
        ours = [r.cost for r in e.solve_batch(qs, [D] * n)]
        for h in fx["reference"]["hop"]:
            if h["k"] == k and h["D"] == D:
                assert ours[: h["n"]] == h["costs"][:n]
        ref = _run("D-TrimCDP", g, gr, qs, k, D=D)
        assert len(ref) == len(qs)
        # D-TrimCDP reports its table's minimum, which is the reference's
        # infinity (100000) when no tree exists, as the engine does
        _compare(ref, ours)
    e.close()
