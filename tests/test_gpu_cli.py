"""The bin/* drivers: reference argument order, input files and result CSV.

Runs each driver on a golden dataset written in the reference formats and
compares the cost column with what the reference programs printed."""
import csv
import os
import subprocess

import numpy as np
import pytest

from gst_b200 import datagen as dg

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpu4gst-1_b200", "bin")


def _rows(path):
    with open(path) as f:
        r = list(csv.reader(f))
    return r[0], [x for x in r[1:] if x]


@pytest.fixture(scope="module")
def dataset(tmp_path_factory, golden):
    fx, g, gr = golden("toy60")
    d = tmp_path_factory.mktemp("cli")
    dg.write_dataset(str(d), "toy", dg.Workload(g, gr, []))
    for k, qs in fx["queries"].items():
        dg.write_queries(str(d / f"toy{k}.csv"), [(np.array(q), -1) for q in qs])
    return fx, str(d) + "/"


@pytest.mark.parametrize("prog,mode", [("TrimCDP", "2"), ("TrimCDP-WB", "1")])
def test_plain_drivers(dataset, prog, mode):
    fx, path = dataset
    n = len(fx["queries"]["3"])
    subprocess.run([os.path.join(BIN, prog), mode, path, "toy", "3", "0", str(n - 1)], check=True,
                   stdout=subprocess.DEVNULL)
    tag = "GPU1_nonHop" if prog == "TrimCDP" else "GPU2_nonHop"
    header, rows = _rows(f"{path}result/exp_{tag}_toy_T3_0-{n - 1}.csv")
    assert header[0] == "task_ID" and header[-2:] == ["counts", "process_num"]
    assert [int(r[3]) for r in rows] == fx["reference"]["prunedpp"]["3"]
    assert [int(r[0]) for r in rows] == list(range(n))


@pytest.mark.parametrize("prog,mode", [("D-TrimCDP", "2"), ("D-TrimCDP-WB", "1")])
def test_diameter_drivers(dataset, prog, mode):
    fx, path = dataset
    for h in fx["reference"]["hop"]:
        if h["k"] != 3:
            continue
        n, D = h["n"], h["D"]
        env = dict(os.environ, GST_ONE_AT_A_TIME="1" if D == 2 else "0")
        subprocess.run([os.path.join(BIN, prog), mode, path, "toy", "3", str(D), "0", str(n - 1)], check=True,
                       stdout=subprocess.DEVNULL, env=env)
        tag = "GPU1_Hop" if prog == "D-TrimCDP" else "GPU2_Hop"
        _, rows = _rows(f"{path}result/exp_{tag}_toy_T3_D{D}_0-{n - 1}.csv")
        assert [int(r[3]) for r in rows] == h["costs"], (prog, D)


def test_driver_errors_are_reported(dataset, tmp_path):
    r = subprocess.run([os.path.join(BIN, "TrimCDP"), "2", str(tmp_path) + "/", "missing", "3", "0", "1"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr
