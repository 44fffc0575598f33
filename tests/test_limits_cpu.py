"""Argument limits of the C ABI that are checked before any device work, so
they run without a GPU: edge offsets must stay below 2^32 (the grow kernel's
edge cursor is a 32-bit unsigned index), vertex ids below 2^31."""
import ctypes

import numpy as np

import gst_b200


def _call_noalloc(lib, V, E):
    dummy = np.zeros(4, np.int64)  # never dereferenced: the call fails first
    ids = np.array([0, 1], np.int32)
    cost = ctypes.c_int64(0)
    root = ctypes.c_int32(0)
    p = dummy.ctypes.data
    return lib.gst_solve_noalloc(V, E, p, p, 2, p, p, ids.ctypes.data, 2, -1, None,
                                 ctypes.byref(cost), ctypes.byref(root))


def test_noalloc_rejects_edge_offsets_from_2_pow_32():
    lib = gst_b200.load_library()
    assert _call_noalloc(lib, 10, 1 << 32) == 6  # GST_E_UNSUPPORTED
    assert b"too large" in lib.gst_last_error()
    assert _call_noalloc(lib, 1 << 31, 10) == 6


def test_noalloc_rejects_null_members():
    lib = gst_b200.load_library()
    dummy = np.zeros(4, np.int64)
    ids = np.array([0, 1], np.int32)
    cost, root = ctypes.c_int64(0), ctypes.c_int32(0)
    p = dummy.ctypes.data
    st = lib.gst_solve_noalloc(10, 10, p, p, 2, p, None, ids.ctypes.data, 2, -1, None,
                               ctypes.byref(cost), ctypes.byref(root))
    assert st == 1  # GST_E_INVALID
