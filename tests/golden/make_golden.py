"""Generates tests/golden/*.json from the reference programs themselves.

Run in a container where the reference sources are mounted and built
(``make -C oracle ref``): every dataset below is regenerated from its seeds,
written in the reference's file formats, and solved by the reference's own
PrunedDP++ and D-PrunedDP++ binaries (oracle/_ref/).  The fixtures store the
generator parameters, a checksum of the generated arrays (so a test can tell
that it regenerated the same inputs) and the costs the reference printed.

    python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "gpu4gst-1_b200"))
sys.path.insert(0, ROOT)

from gst_b200 import datagen as dg  # noqa: E402
import oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def checksum(g, gr) -> str:
    h = hashlib.sha256()
    for a in (g.rowptr, g.col, g.w, gr.ptr, gr.mem):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


# dataset recipes: everything needed to regenerate the inputs
DATASETS = {
    "toy60": dict(graph=dict(V=60, m=2, wmin=1, wmax=20, seed=5, path=False),
                  groups=dict(G=12, seed=7, uniform=[1, 4]),
                  queries=[dict(k=3, n=20, seed=9), dict(k=4, n=10, seed=10)],
                  hop=[dict(k=3, D=D, n=20) for D in (1, 2, 3, 4)] + [dict(k=4, D=2, n=10)]),
    "s3000": dict(graph=dict(V=3000, m=4, wmin=1, wmax=100, seed=3, path=True),
                  groups=dict(G=200, seed=4, geometric=[8, 2, 200]),
                  queries=[dict(k=5, n=12, seed=16), dict(k=7, n=6, seed=18)],
                  hop=[dict(k=5, D=2, n=6), dict(k=5, D=3, n=6),
                       dict(k=7, D=2, n=6), dict(k=7, D=3, n=6), dict(k=7, D=4, n=6)]),
    "c1": dict(graph=dict(V=10000, m=5, wmin=1, wmax=100, seed=1, path=False),
               groups=dict(G=500, seed=101, uniform=[2, 20]),
               queries=[dict(k=3, n=50, seed=201)],
               hop=[dict(k=3, D=3, n=20)]),
    # the C2 benchmark graph and groups (170k vertices, 3,000 groups): parity at full size
    "c2": dict(graph=dict(V=170000, m=20, wmin=1, wmax=100, seed=1, path=True),
               groups=dict(G=3000, seed=101, geometric=[8, 2, 200]),
               queries=[dict(k=5, n=12, seed=201)],
               hop=[dict(k=5, D=4, n=3), dict(k=5, D=5, n=3)]),
}


def build(spec):
    gs = spec["graph"]
    g = dg.ba_graph(gs["V"], gs["m"], gs["wmin"], gs["wmax"], gs["seed"], spanning_path=gs["path"])
    grs = spec["groups"]
    if "uniform" in grs:
        gr = dg.make_groups(g.V, grs["G"], grs["seed"], uniform=tuple(grs["uniform"]))
    else:
        gr = dg.make_groups(g.V, grs["G"], grs["seed"], geometric=tuple(grs["geometric"]))
    queries = {}
    for q in spec["queries"]:
        queries[q["k"]] = [ids.tolist() for ids, _ in dg.make_queries(gr.n, q["n"], q["k"], q["seed"])]
    return g, gr, queries


def edge_case_dataset():
    """A graph with a second component and special groups:
    group 0: vertices 0..2 (main component), group 1: {5}, group 2: {5, 30}
    group 3: only vertices of the second component, group 4: empty,
    group 5: {5} again (vertex 5 covers groups 1, 2, 5)."""
    base = dg.ba_graph(40, 2, 1, 9, 21)
    # second component: a path 40-41-42-43
    V = 44
    edges = []
    for u in range(base.V):
        for j in range(base.rowptr[u], base.rowptr[u + 1]):
            if base.col[j] > u:
                edges.append((u, int(base.col[j]), int(base.w[j])))
    edges += [(40, 41, 3), (41, 42, 4), (42, 43, 5)]
    adj = [[] for _ in range(V)]
    for u, v, w in edges:
        adj[u].append((v, w))
        adj[v].append((u, w))
    rowptr = np.zeros(V + 1, np.int64)
    col, wt = [], []
    for u in range(V):
        adj[u].sort()
        rowptr[u + 1] = rowptr[u] + len(adj[u])
        col += [v for v, _ in adj[u]]
        wt += [w for _, w in adj[u]]
    g = dg.Graph(rowptr, np.array(col, np.int32), np.array(wt, np.int32))
    members = [[0, 1, 2], [5], [5, 30], [41, 43], [], [5], [7, 8, 9, 10]]
    ptr = np.zeros(len(members) + 1, np.int64)
    ptr[1:] = np.cumsum([len(m) for m in members])
    gr = dg.Groups(ptr, np.array(sum(members, []), np.int32))
    queries = {3: [[0, 1, 6], [1, 2, 5], [0, 3, 6], [0, 4, 6], [6, 6, 0], [2, 6, 0]],
               1: [[0], [3], [6]]}
    return g, gr, queries


def run_ref(g, gr, queries, hop_specs, name):
    d = tempfile.mkdtemp(prefix="gstgold_")
    wl = dg.Workload(g, gr, [])
    dg.write_dataset(d, name, wl, binary=False)
    out = {"prunedpp": {}, "hop": []}
    for k, qs in queries.items():
        dg.write_queries(os.path.join(d, f"{name}{k}.csv"), [(np.array(q), -1) for q in qs])
        rows = oracle.run_reference("PrunedDP++", d, name, k, 0, len(qs) - 1)
        out["prunedpp"][str(k)] = [r[3] for r in rows]
    for h in hop_specs:
        k, D, n = h["k"], h["D"], h["n"]
        rows = oracle.run_reference("D-PrunedDP++", d, name, k, 0, n - 1, D=D)
        out["hop"].append(dict(k=k, D=D, n=n, costs=[r[3] for r in rows]))
    return out


def main(names=None):
    for name, spec in DATASETS.items():
        if names and name not in names:
            continue
        g, gr, queries = build(spec)
        res = run_ref(g, gr, queries, spec["hop"], name)
        fx = dict(name=name, spec=spec, checksum=checksum(g, gr),
                  queries={str(k): v for k, v in queries.items()}, reference=res,
                  generated_by="tests/golden/make_golden.py (reference PrunedDP++ / D-PrunedDP++ "
                               "built from source by oracle/Makefile)")
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(fx, f, indent=1)
        print(name, "done")
    if names and "edge" not in names:
        return
    g, gr, queries = edge_case_dataset()
    res = run_ref(g, gr, queries, [dict(k=3, D=2, n=6)], "edge")
    fx = dict(name="edge", checksum=checksum(g, gr),
              graph=dict(rowptr=g.rowptr.tolist(), col=g.col.tolist(), w=g.w.tolist()),
              groups=dict(ptr=gr.ptr.tolist(), mem=gr.mem.tolist()),
              queries={str(k): v for k, v in queries.items()}, reference=res,
              generated_by="tests/golden/make_golden.py")
    with open(os.path.join(HERE, "edge.json"), "w") as f:
        json.dump(fx, f, indent=1)
    print("edge done")


if __name__ == "__main__":
    main(sys.argv[1:])  # dataset names to (re)generate; none: all
