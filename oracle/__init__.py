"""ORACLE -- test infrastructure only.

ctypes binding of the CPU restatement in gst_oracle.cpp, plus runners for
the reference programs built into oracle/_ref/ by oracle/Makefile.  Only
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg
may import this package, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle_gst.so")
REF_DIR = os.path.join(HERE, "_ref")
INF = 100000  # the reference's infinity and infeasible-query cost


class Result(ctypes.Structure):
    _fields_ = [("cost", ctypes.c_longlong), ("feasible", ctypes.c_int), ("root", ctypes.c_int),
                ("n_edges", ctypes.c_int), ("pops", ctypes.c_longlong)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} missing: run `make -C oracle`")
        lib = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        common = [ctypes.c_int64, P, P, P, P, P, ctypes.c_int64, P, ctypes.c_int]
        lib.oracle_prunedpp.argtypes = common + [P, ctypes.c_int, ctypes.POINTER(Result)]
        lib.oracle_dpbf.argtypes = common + [P, ctypes.c_int, ctypes.POINTER(Result)]
        lib.oracle_hop.argtypes = common + [ctypes.c_int, P, ctypes.c_int, ctypes.POINTER(Result)]
        lib.oracle_hop_lean.argtypes = common + [ctypes.c_int, P, ctypes.c_int, ctypes.POINTER(Result)]
        lib.oracle_validate.argtypes = common + [P, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                                 ctypes.c_int]
        for f in (lib.oracle_prunedpp, lib.oracle_dpbf, lib.oracle_hop, lib.oracle_hop_lean,
                  lib.oracle_validate):
            f.restype = ctypes.c_int
        _lib = lib
    return _lib


def _args(graph, groups, query):
    q = np.ascontiguousarray(query, dtype=np.int32)
    return ([graph.V, graph.rowptr.ctypes.data, graph.col.ctypes.data, graph.w.ctypes.data,
             groups.ptr.ctypes.data, groups.mem.ctypes.data, groups.n, q.ctypes.data, len(q)], q)


def _solve(fn, graph, groups, query, extra=()):
    a, keep = _args(graph, groups, query)
    cap = 4096
    while True:
        edges = np.zeros((cap, 3), np.int32)
        r = Result()
        rc = fn(*a, *extra, edges.ctypes.data, cap, ctypes.byref(r))
        if rc != 0:
            raise ValueError("oracle rejected the input")
        if r.n_edges <= cap:
            return r.cost, edges[:r.n_edges].copy(), r.root, r.pops
        cap = r.n_edges


def prunedpp(graph, groups, query):
    """PrunedDP++ restatement; returns (cost, edges[n,3], root, pops)."""
    return _solve(_load().oracle_prunedpp, graph, groups, query)


def dpbf(graph, groups, query):
    """Unpruned exact DPBF; returns (cost, edges, root, pops)."""
    return _solve(_load().oracle_dpbf, graph, groups, query)


def hop(graph, groups, query, D):
    """HOP_cpu restatement (diameter bound D); returns (cost, edges, root, pops)."""
    return _solve(_load().oracle_hop, graph, groups, query, extra=(int(D),))


def hop_lean(graph, groups, query, D):
    """HOP_cpu restatement holding 4 bytes per (vertex, set, hop) state and
    rebuilding the tree from the costs; same answers as hop(), for graphs
    where hop()'s node table does not fit.  Returns (cost, edges, root, pops)."""
    return _solve(_load().oracle_hop_lean, graph, groups, query, extra=(int(D),))


def validate(graph, groups, query, edges, root, cost, D=-1) -> int:
    """0 if `edges` is a tree of weight `cost` touching every queried group with
    hop diameter <= D (D < 0: unbounded); else the failing check's code."""
    a, keep = _args(graph, groups, query)
    e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 3)
    return _load().oracle_validate(*a, e.ctypes.data, len(e), int(root), int(cost), int(D))


# ---- the reference programs ------------------------------------------------

def ref_binary(name: str) -> str:
    return os.path.join(REF_DIR, name)


def run_reference(name: str, dirpath: str, data: str, k: int, start: int, end: int, D=None,
                  mode: int | None = None, timeout: float | None = None) -> list:
    """Runs a reference program with its own argv order and returns the rows
    of the CSV it writes: [(task_id, task, time, cost, memory, counts, process)].

    PrunedDP++ 1 <path> <data> <k> <s> <e>; D-PrunedDP++ 2 <path> <data> <k> <D> <s> <e>
    (code/PrunedDP++/src/main.cpp:16-20, code/D-PrunedDP++/src/main.cpp:16-18)."""
    exe = ref_binary(name)
    path = dirpath.rstrip("/") + "/"
    if mode is None:
        mode = 1 if name == "PrunedDP++" else 2
    argv = [exe, str(mode), path, data, str(k)]
    if D is not None:
        argv.append(str(D))
    argv += [str(start), str(end)]
    subprocess.run(argv, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   timeout=timeout, stdin=subprocess.DEVNULL)
    tag = {"PrunedDP++": "CPU_nonHop", "D-PrunedDP++": "CPU_Hop",
           "TrimCDP": "GPU1_nonHop", "D-TrimCDP": "GPU1_Hop"}[name]
    fn = f"exp_{tag}_{data}_T{k}_" + (f"D{D}_" if D is not None else "") + f"{start}-{end}.csv"
    rows = []
    with open(os.path.join(path, "result", fn)) as f:
        next(f)
        for line in f:
            line = line.strip()
            if not line:
                continue
            p = line.split(",")
            rows.append((int(p[0]), p[1], float(p[2]), int(p[3]), int(p[4]), int(p[5]), int(p[6])))
    return rows
