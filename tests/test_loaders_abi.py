"""Host logic of the C ABI that needs no GPU: the library loads and exports
every entry point of include/gst_b200.h, and the reference-format readers
return what the reference's loaders would (CPU only)."""
import os
import re

import numpy as np
import pytest

import gst_b200
from gst_b200 import datagen as dg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_entry_point():
    lib = gst_b200.load_library()
    with open(os.path.join(ROOT, "include", "gst_b200.h")) as f:
        header = f.read()
    declared = set(re.findall(r"\b(gst_[a-z_]+)\s*\(", header))
    declared -= {"gst_status"}
    assert declared == set(gst_b200.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def _dataset(tmp_path):
    g = dg.ba_graph(300, 3, 1, 40, 17, spanning_path=True)
    gr = dg.make_groups(g.V, 25, 18, uniform=(1, 6))
    qs = dg.make_queries(gr.n, 7, 4, 19)
    wl = dg.Workload(g, gr, qs)
    dg.write_dataset(str(tmp_path), "tiny", wl)
    return g, gr, qs


def test_text_graph_reader_matches_generator(tmp_path):
    g, _, _ = _dataset(tmp_path)
    c = gst_b200.read_input_graph(str(tmp_path / "tiny.in"))
    assert c.V == g.V and c.E == g.E
    np.testing.assert_array_equal(c.rowptr, g.rowptr)
    np.testing.assert_array_equal(c.col, g.col)
    np.testing.assert_array_equal(c.w, g.w)


def test_binary_csr_reader_matches_generator(tmp_path):
    g, _, _ = _dataset(tmp_path)
    c = gst_b200.read_binary_csr(str(tmp_path / "tiny"))
    np.testing.assert_array_equal(c.rowptr, g.rowptr)
    np.testing.assert_array_equal(c.col, g.col)
    np.testing.assert_array_equal(c.w, g.w)


def test_group_and_query_readers(tmp_path):
    _, gr, qs = _dataset(tmp_path)
    ptr, mem = gst_b200.read_groups(str(tmp_path / "tiny.g"))
    np.testing.assert_array_equal(ptr, gr.ptr)
    np.testing.assert_array_equal(mem, gr.mem)
    got = gst_b200.read_queries(str(tmp_path / "tiny4.csv"))
    assert [q.tolist() for q in got] == [q.tolist() for q, _ in qs]


def test_reader_quirks(tmp_path):
    # both directions stored, rows sorted by (neighbour, weight), lines that do not
    # hold three fields skipped, CRLF and trailing spaces tolerated (the reference
    # splits on single spaces and would drop the line with a trailing space)
    p = tmp_path / "q.in"
    p.write_text("4 3\r\n2 0 5\r\n1 0 7 \r\n0 3\r\n3 1 2\n")
    c = gst_b200.read_input_graph(str(p))
    assert c.V == 4
    assert c.col[c.rowptr[0]:c.rowptr[1]].tolist() == [1, 2]
    assert c.w[c.rowptr[0]:c.rowptr[1]].tolist() == [7, 5]
    assert c.col[c.rowptr[1]:c.rowptr[2]].tolist() == [0, 3]
    g = tmp_path / "q.g"
    g.write_text("g2:3 1 \ng1:2\n\ng4:\n")
    ptr, mem = gst_b200.read_groups(str(g))
    assert ptr.tolist() == [0, 1, 3, 3, 3]
    assert mem.tolist() == [2, 1, 3]
    q = tmp_path / "q3.csv"
    q.write_text("0 1 3 \n\n2 2 0\n")
    assert [x.tolist() for x in gst_b200.read_queries(str(q))] == [[0, 1, 3], [2, 2, 0]]


def test_readers_fail_with_status_not_exit(tmp_path):
    with pytest.raises(gst_b200.GstError) as e:
        gst_b200.read_input_graph(str(tmp_path / "missing.in"))
    assert e.value.status == 2  # GST_E_IO
    bad = tmp_path / "bad.in"
    bad.write_text("3\n0 5 1\n")
    with pytest.raises(gst_b200.GstError) as e:
        gst_b200.read_input_graph(str(bad))
    assert e.value.status == 3  # GST_E_FORMAT: endpoint out of range
    badg = tmp_path / "bad.g"
    badg.write_text("x1:1 2\n")
    with pytest.raises(gst_b200.GstError):
        gst_b200.read_groups(str(badg))
    with pytest.raises(gst_b200.GstError) as e:
        gst_b200.read_binary_csr(str(tmp_path / "nothing"))
    assert e.value.status == 2


def test_engine_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gst_b200.GstError) as e:
        gst_b200.Engine()
    assert e.value.status == 4  # GST_E_CUDA
