"""Python binding of the B200 group Steiner tree engine (libgst_b200.so).

A thin ctypes layer over the C ABI in include/gst_b200.h; it adds no
computation of its own.  The library must be built in-tree
(``__graft_entry__.build()`` or ``make -C gpu4gst-1_b200``); importing the
engine API without it raises, there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libgst_b200.so")

GST_OK = 0
STATUS = {0: "GST_OK", 1: "GST_E_INVALID", 2: "GST_E_IO", 3: "GST_E_FORMAT", 4: "GST_E_CUDA",
          5: "GST_E_NOMEM", 6: "GST_E_UNSUPPORTED", 7: "GST_E_LIMIT", 8: "GST_E_STATE",
          9: "GST_E_TIMEOUT"}
# statuses that describe one query's outcome (returned in Result.status)
# rather than a failed call: GST_OK, GST_E_NOMEM (does not fit the arena),
# GST_E_LIMIT (a device-side bound was hit)
PER_QUERY = (0, 5, 7)
MAX_K = 7
MAX_D = 15
REF_INF = 100000

# every entry point include/gst_b200.h declares
EXPORTS = [
    "gst_last_error", "gst_read_input_graph", "gst_read_binary_csr", "gst_read_groups",
    "gst_read_queries", "gst_csr_free", "gst_groups_free", "gst_queries_free",
    "gst_engine_create", "gst_engine_destroy", "gst_engine_load_graph", "gst_engine_load_groups",
    "gst_result_free", "gst_solve", "gst_solve_batch", "gst_server_start", "gst_server_submit",
    "gst_server_wait", "gst_server_stop", "gst_engine_profile", "gst_solve_noalloc", "gst_sizeof",
    "gst_engine_set_tuning", "gst_engine_get_tuning",
]


class GstError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class _Csr(ctypes.Structure):
    _fields_ = [("V", ctypes.c_int64), ("E", ctypes.c_int64), ("rowptr", ctypes.POINTER(ctypes.c_int64)),
                ("col", ctypes.POINTER(ctypes.c_int32)), ("w", ctypes.POINTER(ctypes.c_int32))]


class _Groups(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("ptr", ctypes.POINTER(ctypes.c_int64)),
                ("members", ctypes.POINTER(ctypes.c_int32))]


class _Queries(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("ptr", ctypes.POINTER(ctypes.c_int64)),
                ("ids", ctypes.POINTER(ctypes.c_int32))]


class _Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("arena_fraction", ctypes.c_double),
                ("arena_bytes", ctypes.c_int64), ("max_slots", ctypes.c_int),
                ("rounds_per_poll", ctypes.c_int), ("max_rounds", ctypes.c_int),
                ("profile", ctypes.c_int), ("bucket_shift", ctypes.c_int)]


class _Profile(ctypes.Structure):
    _fields_ = [("run_ms", ctypes.c_double), ("grow_ms", ctypes.c_double),
                ("grow_launches", ctypes.c_int64), ("merge_ms", ctypes.c_double),
                ("merge_launches", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("rounds", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64)]


class _Tuning(ctypes.Structure):
    _fields_ = [("grow_lanes", ctypes.c_int), ("rounds_per_poll", ctypes.c_int), ("max_slots", ctypes.c_int),
                ("chunk_pairs", (ctypes.c_int * 2) * (MAX_K + 1)), ("bucket_mult", ctypes.c_int * (MAX_K + 1)),
                ("overlap", ctypes.c_int)]


class _Stats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int64), ("frontier", ctypes.c_int64), ("relax", ctypes.c_int64),
                ("improve", ctypes.c_int64), ("merges", ctypes.c_int64), ("merge_items", ctypes.c_int64),
                ("merge_passed", ctypes.c_int64), ("touched", ctypes.c_int64),
                ("device_ms", ctypes.c_double), ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double)]


class _Result(ctypes.Structure):
    _fields_ = [("cost", ctypes.c_int64), ("feasible", ctypes.c_int32), ("root", ctypes.c_int32),
                ("n_edges", ctypes.c_int32), ("edges", ctypes.POINTER(ctypes.c_int32)), ("stats", _Stats)]


_lib = None


def load_library() -> ctypes.CDLL:
    """Loads libgst_b200.so; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built: the CUDA engine is required "
                           "(run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    lib.gst_last_error.restype = ctypes.c_char_p
    lib.gst_read_input_graph.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Csr)]
    lib.gst_read_binary_csr.argtypes = [ctypes.c_char_p] * 3 + [ctypes.POINTER(_Csr)]
    lib.gst_read_groups.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Groups)]
    lib.gst_read_queries.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Queries)]
    lib.gst_csr_free.argtypes = [ctypes.POINTER(_Csr)]
    lib.gst_groups_free.argtypes = [ctypes.POINTER(_Groups)]
    lib.gst_queries_free.argtypes = [ctypes.POINTER(_Queries)]
    for f in (lib.gst_csr_free, lib.gst_groups_free, lib.gst_queries_free):
        f.restype = None
    lib.gst_engine_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(P)]
    lib.gst_engine_destroy.argtypes = [P]
    lib.gst_engine_destroy.restype = None
    lib.gst_engine_load_graph.argtypes = [P, ctypes.c_int64, P, P, P]
    lib.gst_engine_load_groups.argtypes = [P, ctypes.c_int64, P, P]
    lib.gst_result_free.argtypes = [ctypes.POINTER(_Result)]
    lib.gst_result_free.restype = None
    lib.gst_solve.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Result)]
    lib.gst_solve_batch.argtypes = [P, ctypes.c_int64, P, P, P, P, P]
    lib.gst_server_start.argtypes = [P, ctypes.POINTER(P)]
    lib.gst_server_submit.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
    lib.gst_server_wait.argtypes = [P, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(_Result)]
    lib.gst_solve_noalloc.argtypes = [ctypes.c_int64, ctypes.c_int64, P, P, ctypes.c_int64, P, P, P,
                                      ctypes.c_int, ctypes.c_int, P, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int32)]
    lib.gst_solve_noalloc.restype = ctypes.c_int
    lib.gst_engine_set_tuning.argtypes = [P, ctypes.POINTER(_Tuning)]
    lib.gst_engine_set_tuning.restype = ctypes.c_int
    lib.gst_engine_get_tuning.argtypes = [P, ctypes.POINTER(_Tuning)]
    lib.gst_engine_get_tuning.restype = ctypes.c_int
    lib.gst_engine_profile.argtypes = [P, ctypes.POINTER(_Profile)]
    lib.gst_engine_profile.restype = ctypes.c_int
    lib.gst_server_stop.argtypes = [P]
    lib.gst_server_stop.restype = None
    for name in ("gst_read_input_graph", "gst_read_binary_csr", "gst_read_groups", "gst_read_queries",
                 "gst_engine_create", "gst_engine_load_graph", "gst_engine_load_groups", "gst_solve",
                 "gst_solve_batch", "gst_server_start", "gst_server_submit", "gst_server_wait"):
        getattr(lib, name).restype = ctypes.c_int
    lib.gst_sizeof.argtypes = [ctypes.c_char_p]
    lib.gst_sizeof.restype = ctypes.c_int64
    # the structs below must be laid out as the library was compiled
    for cname, py in (("gst_result", _Result), ("gst_stats", _Stats), ("gst_engine_config", _Config),
                      ("gst_profile", _Profile), ("gst_tuning", _Tuning), ("gst_csr", _Csr), ("gst_groups", _Groups),
                      ("gst_queries", _Queries)):
        n = lib.gst_sizeof(cname.encode())
        if n != ctypes.sizeof(py):
            raise RuntimeError(f"{LIB_PATH}: sizeof({cname}) is {n}, the binding expects "
                               f"{ctypes.sizeof(py)}; rebuild the library")
    _lib = lib
    return lib


def _check(status: int, what: str = "") -> None:
    if status != GST_OK:
        msg = load_library().gst_last_error().decode(errors="replace")
        raise GstError(status, f"{what}: {msg}" if what else msg)


# ---- readers (reference formats) -------------------------------------------

@dataclass
class Csr:
    rowptr: np.ndarray
    col: np.ndarray
    w: np.ndarray

    @property
    def V(self) -> int:
        return len(self.rowptr) - 1

    @property
    def E(self) -> int:
        return int(self.rowptr[-1])


def read_input_graph(path: str) -> Csr:
    lib, c = load_library(), _Csr()
    _check(lib.gst_read_input_graph(path.encode(), ctypes.byref(c)), path)
    try:
        return Csr(np.ctypeslib.as_array(c.rowptr, (c.V + 1,)).copy(),
                   np.ctypeslib.as_array(c.col, (max(c.E, 1),))[:c.E].copy(),
                   np.ctypeslib.as_array(c.w, (max(c.E, 1),))[:c.E].copy())
    finally:
        lib.gst_csr_free(ctypes.byref(c))


def read_binary_csr(prefix: str) -> Csr:
    lib, c = load_library(), _Csr()
    _check(lib.gst_read_binary_csr((prefix + "_beg_pos.bin").encode(), (prefix + "_csr.bin").encode(),
                                   (prefix + "_weight.bin").encode(), ctypes.byref(c)), prefix)
    try:
        return Csr(np.ctypeslib.as_array(c.rowptr, (c.V + 1,)).copy(),
                   np.ctypeslib.as_array(c.col, (max(c.E, 1),))[:c.E].copy(),
                   np.ctypeslib.as_array(c.w, (max(c.E, 1),))[:c.E].copy())
    finally:
        lib.gst_csr_free(ctypes.byref(c))


def read_groups(path: str):
    lib, g = load_library(), _Groups()
    _check(lib.gst_read_groups(path.encode(), ctypes.byref(g)), path)
    try:
        ptr = np.ctypeslib.as_array(g.ptr, (g.n + 1,)).copy()
        m = int(ptr[-1])
        mem = np.ctypeslib.as_array(g.members, (max(m, 1),))[:m].copy()
        return ptr, mem
    finally:
        lib.gst_groups_free(ctypes.byref(g))


def read_queries(path: str) -> list:
    lib, q = load_library(), _Queries()
    _check(lib.gst_read_queries(path.encode(), ctypes.byref(q)), path)
    try:
        ptr = np.ctypeslib.as_array(q.ptr, (q.n + 1,)).copy()
        m = int(ptr[-1])
        ids = np.ctypeslib.as_array(q.ids, (max(m, 1),))[:m].copy()
        return [ids[ptr[i]:ptr[i + 1]].copy() for i in range(q.n)]
    finally:
        lib.gst_queries_free(ctypes.byref(q))


# ---- engine -------------------------------------------------------------------

@dataclass
class Result:
    cost: int
    feasible: bool
    root: int
    edges: np.ndarray  # (n, 3) int32: u, v, w
    stats: dict
    status: int = GST_OK


def _take_result(lib, r: _Result, status: int) -> Result:
    n = r.n_edges
    edges = np.zeros((0, 3), np.int32)
    if n and r.edges:
        edges = np.ctypeslib.as_array(r.edges, (n * 3,)).reshape(n, 3).copy()
    st = {f: getattr(r.stats, f) for f, _ in _Stats._fields_}
    out = Result(int(r.cost), bool(r.feasible), int(r.root), edges, st, status)
    lib.gst_result_free(ctypes.byref(r))
    return out


class Engine:
    """One engine per device: graph + groups resident in HBM, arena for tables."""

    def __init__(self, device: int = 0, arena_fraction: float = 0.0, arena_bytes: int = 0,
                 max_slots: int = 0, rounds_per_poll: int = 0, max_rounds: int = 0,
                 profile: bool = False, bucket_shift: int = 0):
        self._lib = load_library()
        cfg = _Config(device, arena_fraction, arena_bytes, max_slots, rounds_per_poll, max_rounds,
                      1 if profile else 0, bucket_shift)
        h = ctypes.c_void_p()
        _check(self._lib.gst_engine_create(ctypes.byref(cfg), ctypes.byref(h)), "engine_create")
        self._h = h
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gst_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_graph(self, rowptr, col, w):
        rowptr = np.ascontiguousarray(rowptr, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        w = np.ascontiguousarray(w, np.int32)
        _check(self._lib.gst_engine_load_graph(self._h, len(rowptr) - 1, rowptr.ctypes.data,
                                               col.ctypes.data, w.ctypes.data), "load_graph")

    def load_groups(self, ptr, members):
        ptr = np.ascontiguousarray(ptr, np.int64)
        members = np.ascontiguousarray(members, np.int32)
        _check(self._lib.gst_engine_load_groups(self._h, len(ptr) - 1, ptr.ctypes.data,
                                                members.ctypes.data), "load_groups")

    def solve(self, group_ids, D: int = -1) -> Result:
        ids = np.ascontiguousarray(group_ids, np.int32)
        r = _Result()
        st = self._lib.gst_solve(self._h, ids.ctypes.data, len(ids), int(D), ctypes.byref(r))
        if st not in PER_QUERY:
            _check(st, "solve")
        return _take_result(self._lib, r, st)

    def solve_batch(self, queries, Ds=None) -> list:
        n = len(queries)
        ptr = np.zeros(n + 1, np.int64)
        ptr[1:] = np.cumsum([len(q) for q in queries])
        ids = np.concatenate([np.asarray(q, np.int32) for q in queries]) if n else np.zeros(1, np.int32)
        ids = np.ascontiguousarray(ids, np.int32)
        Darr = None if Ds is None else np.ascontiguousarray(Ds, np.int32)
        res = (_Result * max(n, 1))()
        sts = np.zeros(max(n, 1), np.int32)
        _check(self._lib.gst_solve_batch(self._h, n, ptr.ctypes.data, ids.ctypes.data,
                                         None if Darr is None else Darr.ctypes.data, res,
                                         sts.ctypes.data), "solve_batch")
        return [_take_result(self._lib, res[i], int(sts[i])) for i in range(n)]

    def profile(self) -> dict:
        """Device measurements of the last solve / solve_batch call."""
        p = _Profile()
        _check(self._lib.gst_engine_profile(self._h, ctypes.byref(p)), "profile")
        return {f: getattr(p, f) for f, _ in _Profile._fields_}

    def get_tuning(self) -> dict:
        """Launch and scheduling parameters (gst_tuning) as a dict:
        grow_lanes, rounds_per_poll, max_slots, chunk_pairs[k] = [plain, D],
        bucket_mult[k], overlap (1 serial, 2 merge and grow on two streams)."""
        t = _Tuning()
        _check(self._lib.gst_engine_get_tuning(self._h, ctypes.byref(t)), "get_tuning")
        return {"grow_lanes": t.grow_lanes, "rounds_per_poll": t.rounds_per_poll, "max_slots": t.max_slots,
                "chunk_pairs": [[t.chunk_pairs[k][0], t.chunk_pairs[k][1]] for k in range(MAX_K + 1)],
                "bucket_mult": [t.bucket_mult[k] for k in range(MAX_K + 1)], "overlap": t.overlap}

    def set_tuning(self, tuning: dict) -> None:
        """Sets the parameters present in `tuning` (same keys as get_tuning;
        absent or 0 keeps the current value)."""
        t = _Tuning()
        t.grow_lanes = int(tuning.get("grow_lanes", 0))
        t.rounds_per_poll = int(tuning.get("rounds_per_poll", 0))
        t.max_slots = int(tuning.get("max_slots", 0))
        t.overlap = int(tuning.get("overlap", 0))
        for k, pair in enumerate(tuning.get("chunk_pairs", [])[: MAX_K + 1]):
            t.chunk_pairs[k][0], t.chunk_pairs[k][1] = int(pair[0]), int(pair[1])
        for k, m in enumerate(tuning.get("bucket_mult", [])[: MAX_K + 1]):
            t.bucket_mult[k] = int(m)
        _check(self._lib.gst_engine_set_tuning(self._h, ctypes.byref(t)), "set_tuning")

    def load_tuning(self, path: str) -> dict:
        """Applies a parameter file written by gst_b200.autotune; returns the
        tuning it set."""
        from .autotune import load
        t = load(path)
        self.set_tuning(t)
        return t

    def server(self) -> "Server":
        return Server(self)


class Server:
    """Continuous-batching request loop over an engine."""

    def __init__(self, engine: Engine):
        self._e = engine
        self._lib = engine._lib
        h = ctypes.c_void_p()
        _check(self._lib.gst_server_start(engine._h, ctypes.byref(h)), "server_start")
        self._h = h

    def submit(self, group_ids, D: int = -1) -> int:
        ids = np.ascontiguousarray(group_ids, np.int32)
        t = ctypes.c_uint64()
        _check(self._lib.gst_server_submit(self._h, ids.ctypes.data, len(ids), int(D), ctypes.byref(t)),
               "submit")
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> Result:
        r = _Result()
        st = self._lib.gst_server_wait(self._h, ticket, float(timeout_ms), ctypes.byref(r))
        if st not in PER_QUERY:
            _check(st, "wait")
        return _take_result(self._lib, r, st)

    def stop(self):
        if self._h:
            self._lib.gst_server_stop(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()
