"""The engine's bound on device waits (GST_WATCHDOG_S), exercised without a
GPU fault: a child process sets the bound far below one poll of the device
rounds, so its first solve must come back with GST_E_CUDA and the watchdog
message instead of blocking, later calls must be refused, and the process must
still exit normally (the unfinished device work ends with its context).  It
runs in a child so that the refused engine, which frees nothing, does not
hold memory for the other tests."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
import gst_b200
from gst_b200 import datagen as dg
g = dg.ba_graph(50000, 5, 1, 100, seed=5)
gr = dg.make_groups(g.V, 300, seed=6, uniform=(2, 10))
e = gst_b200.Engine(device=0, arena_bytes=2 << 30)
e.load_graph(g.rowptr, g.col, g.w)
e.load_groups(gr.ptr, gr.mem)
try:
    e.solve([0, 1, 2, 3, 4, 5, 6], 4)
    print("FIRST-FINISHED")
except gst_b200.GstError as x:
    print("FIRST-ERROR", x)
try:
    e.solve([0, 1, 2])
    print("SECOND-FINISHED")
except gst_b200.GstError as x:
    print("SECOND-ERROR", x)
e.close()
print("EXIT")
"""


def test_a_device_wait_beyond_the_bound_fails_the_call_instead_of_blocking():
    env = dict(os.environ, GST_WATCHDOG_S="0.0001")
    r = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "gpu4gst-1_b200")],
                       capture_output=True, text=True, env=env, timeout=600)
    out = r.stdout
    assert r.returncode == 0, r.stderr[-2000:]
    assert "FIRST-ERROR" in out and "did not finish" in out, out
    assert "SECOND-ERROR" in out and "unusable" in out, out
    assert "EXIT" in out
