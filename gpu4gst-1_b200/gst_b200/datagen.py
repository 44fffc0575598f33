"""Seeded synthetic GST workloads in the reference's file formats.

The reference is benchmarked on external social graphs that are not available
here; Barabasi-Albert power-law graphs of the same shapes stand in for them.
The graph itself is built by ``libgst_datagen.so`` (C++, fast enough for 4M
vertices); groups and queries are drawn here with numpy.

Formats written (all read by the reference and by this engine's loaders):

* ``<data>.in``  -- "V E" then "u v w" per undirected edge
  (code/PrunedDP++/include/graph_hash_of_mixed_weighted_read_for_GSTP.h:15-66)
* ``<data>_beg_pos.bin`` / ``_csr.bin`` / ``_weight.bin`` -- int64 CSR
  (code/TrimCDP-WB/include/graph.hpp:12-118)
* ``<data>.g``   -- lines "gK:v v v", K 1-based (same file :116-171)
* ``<data><k>.csv`` -- lines of k 0-based group ids (same file :172-218)
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_DIR = os.path.join(os.path.dirname(_HERE), "lib")
_lib = None


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(_LIB_DIR, "libgst_datagen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built; run __graft_entry__.build()")
        lib = ctypes.CDLL(path)
        i64, i32p, i64p = ctypes.c_int64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)
        lib.gstgen_ba.argtypes = [i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
        lib.gstgen_ba.restype = ctypes.c_int
        lib.gstgen_num_vertices.argtypes = [ctypes.c_void_p]
        lib.gstgen_num_vertices.restype = i64
        lib.gstgen_num_arcs.argtypes = [ctypes.c_void_p]
        lib.gstgen_num_arcs.restype = i64
        lib.gstgen_copy_csr.argtypes = [ctypes.c_void_p, i64p, i32p, i32p]
        lib.gstgen_copy_csr.restype = ctypes.c_int
        lib.gstgen_free.argtypes = [ctypes.c_void_p]
        lib.gstgen_free.restype = None
        lib.gstgen_write_in.argtypes = [ctypes.c_char_p, i64, i64p, i32p, i32p]
        lib.gstgen_write_in.restype = ctypes.c_int
        lib.gstgen_write_bin.argtypes = [ctypes.c_char_p, i64, i64p, i32p, i32p]
        lib.gstgen_write_bin.restype = ctypes.c_int
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


@dataclass
class Graph:
    """Undirected graph as CSR with both directions stored, rows sorted."""
    rowptr: np.ndarray  # int64, V+1
    col: np.ndarray     # int32, E
    w: np.ndarray       # int32, E

    @property
    def V(self) -> int:
        return len(self.rowptr) - 1

    @property
    def E(self) -> int:
        return int(self.rowptr[-1])


@dataclass
class Groups:
    ptr: np.ndarray  # int64, G+1
    mem: np.ndarray  # int32

    @property
    def n(self) -> int:
        return len(self.ptr) - 1

    def members(self, g: int) -> np.ndarray:
        return self.mem[self.ptr[g]:self.ptr[g + 1]]


@dataclass
class Workload:
    graph: Graph
    groups: Groups
    queries: list = field(default_factory=list)  # list of (group_ids ndarray, D) ; D=-1 unbounded


def ba_graph(V: int, m: int, wmin: int, wmax: int, seed: int, spanning_path: bool = False) -> Graph:
    lib = _load()
    h = ctypes.c_void_p()
    rc = lib.gstgen_ba(V, m, wmin, wmax, 1 if spanning_path else 0, seed, ctypes.byref(h))
    if rc != 0:
        raise ValueError("bad BA parameters")
    try:
        E = lib.gstgen_num_arcs(h)
        rowptr = np.empty(V + 1, np.int64)
        col = np.empty(E, np.int32)
        w = np.empty(E, np.int32)
        lib.gstgen_copy_csr(h, _p(rowptr, ctypes.c_int64), _p(col, ctypes.c_int32), _p(w, ctypes.c_int32))
    finally:
        lib.gstgen_free(h)
    return Graph(rowptr, col, w)


def make_groups(V: int, G: int, seed: int, *, uniform=None, geometric=None) -> Groups:
    """G groups of uniformly random distinct vertices.

    uniform=(a, b): sizes uniform in [a, b];
    geometric=(mean, lo, hi): sizes geometric on {1,2,..} with that mean, clipped.
    """
    rng = np.random.default_rng(seed)
    if uniform is not None:
        sizes = rng.integers(uniform[0], uniform[1] + 1, size=G)
    else:
        mean, lo, hi = geometric
        sizes = np.clip(rng.geometric(1.0 / mean, size=G), lo, hi)
    sizes = np.minimum(sizes, V)
    ptr = np.zeros(G + 1, np.int64)
    ptr[1:] = np.cumsum(sizes)
    mem = np.empty(int(ptr[-1]), np.int32)
    for g in range(G):
        s = int(sizes[g])
        got = np.unique(rng.integers(0, V, size=2 * s + 8))
        while len(got) < s:
            got = np.unique(np.concatenate([got, rng.integers(0, V, size=2 * s + 8)]))
        pick = rng.permutation(got)[:s]
        mem[ptr[g]:ptr[g + 1]] = np.sort(pick)
    return Groups(ptr, mem)


def make_queries(G: int, n: int, k, seed: int, D=-1) -> list:
    """n queries of distinct group ids.  k: int or sequence to draw from
    (with optional probabilities as (values, probs)); D: int, or a callable
    rng -> int per query."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        if isinstance(k, int):
            kk = k
        elif isinstance(k, tuple) and len(k) == 2 and not isinstance(k[0], int):
            kk = int(rng.choice(k[0], p=k[1]))
        else:
            kk = int(rng.choice(k))
        ids = rng.choice(G, size=kk, replace=False).astype(np.int32)
        d = D(rng) if callable(D) else D
        out.append((ids, int(d)))
    return out


# ---- the workloads the reference's experiments are sized on ----------------

def config_c1(seed: int = 1) -> Workload:
    """BA V=10,000 m=5 w~U[1,100]; 500 groups U[2,20]; 50 queries k=3."""
    g = ba_graph(10_000, 5, 1, 100, seed)
    gr = make_groups(g.V, 500, seed + 100, uniform=(2, 20))
    return Workload(g, gr, make_queries(gr.n, 50, 3, seed + 200))


def config_c2(seed: int = 1, n_queries: int = 300) -> Workload:
    """BA V=170,000 m=20 + spanning path, w~U[1,100]; 3,000 groups Geom(8) in
    [2,200]; 300 queries of k=5."""
    g = ba_graph(170_000, 20, 1, 100, seed, spanning_path=True)
    gr = make_groups(g.V, 3000, seed + 100, geometric=(8, 2, 200))
    return Workload(g, gr, make_queries(gr.n, n_queries, 5, seed + 200))


def config_c3(seed: int = 1, n_queries: int = 300) -> Workload:
    """BA V=1,000,000 m=10, w~U[1,1000]; 10,000 groups Geom(10) in [2,500];
    300 queries of k=7 with D uniform in {2,3,4,5}."""
    g = ba_graph(1_000_000, 10, 1, 1000, seed)
    gr = make_groups(g.V, 10_000, seed + 100, geometric=(10, 2, 500))
    return Workload(g, gr, make_queries(gr.n, n_queries, 7, seed + 200,
                                        D=lambda r: int(r.integers(2, 6))))


def config_c4(seed: int = 1, n_queries: int = 300) -> Workload:
    """BA V=4,000,000 m=9 + spanning path, w~U[1,100]; 20,000 groups Geom(12)
    in [2,1000]; 300 queries, k uniform in {3,5,7}, D unbounded for half and
    uniform in [2,5] for the rest."""
    g = ba_graph(4_000_000, 9, 1, 100, seed, spanning_path=True)
    gr = make_groups(g.V, 20_000, seed + 100, geometric=(12, 2, 1000))
    return Workload(g, gr, make_queries(gr.n, n_queries, [3, 5, 7], seed + 200,
                                        D=lambda r: -1 if r.random() < 0.5 else int(r.integers(2, 6))))


# ---- writers ----------------------------------------------------------------

def write_in(path: str, g: Graph) -> None:
    rc = _load().gstgen_write_in(path.encode(), g.V, _p(g.rowptr, ctypes.c_int64),
                                 _p(g.col, ctypes.c_int32), _p(g.w, ctypes.c_int32))
    if rc != 0:
        raise OSError(f"cannot write {path}")


def write_bin(prefix: str, g: Graph) -> None:
    rc = _load().gstgen_write_bin(prefix.encode(), g.V, _p(g.rowptr, ctypes.c_int64),
                                  _p(g.col, ctypes.c_int32), _p(g.w, ctypes.c_int32))
    if rc != 0:
        raise OSError(f"cannot write {prefix}_*.bin")


def write_groups(path: str, gr: Groups) -> None:
    with open(path, "w") as f:
        for gi in range(gr.n):
            f.write(f"g{gi + 1}:" + " ".join(map(str, gr.members(gi).tolist())) + "\n")


def write_queries(path: str, queries) -> None:
    with open(path, "w") as f:
        for ids, _d in queries:
            f.write(" ".join(map(str, [int(x) for x in ids])) + "\n")


def write_dataset(dirpath: str, name: str, wl: Workload, *, text=True, binary=True) -> None:
    """Writes every reference input file for `wl` under dirpath (with a
    trailing result/ directory, which the reference programs write into).
    Queries are grouped by k into <name><k>.csv."""
    os.makedirs(os.path.join(dirpath, "result"), exist_ok=True)
    base = os.path.join(dirpath, name)
    if text:
        write_in(base + ".in", wl.graph)
    if binary:
        write_bin(base, wl.graph)
    write_groups(base + ".g", wl.groups)
    byk = {}
    for q in wl.queries:
        byk.setdefault(len(q[0]), []).append(q)
    for k, qs in byk.items():
        write_queries(f"{base}{k}.csv", qs)
