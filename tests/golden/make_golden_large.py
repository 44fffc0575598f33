"""Generates tests/golden/c3.json, c4.json and c2_batch.json: reference
costs at the benchmark sizes, from the reference programs themselves.

C2_batch is the 170k-vertex k=5 workload's whole 300-query batch (BA m=20 +
spanning path, w U[1,100], 3,000 groups Geom(8) in [2,200]), every query
pinned by PrunedDP++.

C3 is the 1M-vertex diameter-bounded k=7 workload (BA m=10, w U[1,1000],
10,000 groups Geom(10) in [2,500], 300 queries with D in {2..5}); C4 is the
4M-vertex mixed workload the benchmark's headline is measured on (BA m=9 +
spanning path, w U[1,100], 20,000 groups Geom(12) in [2,1000], 300 queries,
k in {3,5,7}, half D-bounded).  Both are regenerated from their seeds by the
project's generator; the fixtures store the query indices of a seeded subset
of each (k, D) cell, the queries themselves and the costs the reference
printed.

The reference programs (oracle/_ref/, built by oracle/Makefile) run as many
single-threaded processes at once as the cores and a memory budget allow:
D-PrunedDP++ allocates its whole (vertex, group set, depth) table up front
(44-byte nodes in nested vectors, code/D-PrunedDP++/include/CPUHOP.h:107-130),
so its memory is known before it starts.  Cells whose table does not fit
(C4 k=7 with a diameter bound: 88 to 155 GB) are recorded as not pinned,
with the reason.  Every finished cell is written to the fixture at once, so
an interrupted run keeps what it finished and a rerun resumes.

With --restatement, the cells the reference cannot run are pinned instead by
oracle.hop_lean, the restatement of the reference's HOP_cpu that holds 4
bytes per (vertex, set, hop) state (12 GB for k=7, D=5 on 4M vertices); it
equals D-PrunedDP++ on every C3 cell and on the small fixtures.  Such cells
name that program in "program", so a reader (and the benchmark's parity
line) can tell them from cells the reference binaries printed.

    python tests/golden/make_golden_large.py c4|c3|c2 [--procs N] [--mem-gb G] [--restatement]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu4gst-1_b200"))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from gst_b200 import datagen as dg  # noqa: E402
import make_golden as mg  # noqa: E402
import oracle  # noqa: E402

# Seeded subsets: the first n queries (in workload order) of each (k, D)
# cell, D = -1 for plain.  n is set by what the reference finishes in
# reasonable time on a few cores; 0 marks a cell the reference cannot run.
SUBSETS = {
    "c4": {(3, -1): 52, (5, -1): 51, (7, -1): 24,
           (3, 2): 10, (3, 3): 10, (3, 4): 12, (3, 5): 12,
           (5, 2): 6, (5, 3): 6, (5, 4): 6, (5, 5): 6,
           (7, 2): 0, (7, 3): 0, (7, 4): 0, (7, 5): 0},
    "c3": {(7, 2): 10, (7, 3): 10, (7, 4): 6, (7, 5): 6},
    "c2": {(5, -1): 300},
}
# The C2 batch fixture is written beside the older tests/golden/c2.json (its
# first 12 queries, in make_golden.py's format), not over it.
FIXTURE_FILE = {"c2": "c2_batch"}
# Cells pinned by the restatement (--restatement): the first n queries of
# each cell the reference cannot run.
LEAN_SUBSETS = {"c4": {(7, 2): 14, (7, 3): 11, (7, 4): 10, (7, 5): 13}}
LEAN_PROGRAM = "oracle.hop_lean"
PLAIN_PER_JOB = 4  # plain queries per process (amortises the graph load)


def workload(name):
    if name == "c4":
        return dg.config_c4(1, n_queries=300), dict(config="c4", seed=1, n_queries=300)
    if name == "c2":
        return dg.config_c2(1, n_queries=300), dict(config="c2", seed=1, n_queries=300)
    if name == "c3":
        return dg.config_c3(1, n_queries=300), dict(config="c3", seed=1, n_queries=300)
    raise SystemExit(f"unknown dataset {name}")


def mem_bytes(wl, k, D):
    """Resident memory of one reference process: the graph in its hash and
    vector forms (measured about 2 GB for C4), plus D-PrunedDP++'s table of
    V * 2^k * (D+1) nodes of 44 bytes in vectors (24-byte header and a
    16-byte allocation per (v, set))."""
    g = 2.5e9 * wl.graph.E / 80e6 + 0.3e9
    if D < 0:
        return g
    return g + wl.graph.V * (1 << k) * (40 + 44 * (D + 1))


def lean_mem_bytes(wl, k, D):
    """Resident memory of one restatement process: the graph arrays (mapped),
    the int32 cost table and its heap (measured under a fifth of the table
    for C4 k=7 D=5; budgeted at a quarter)."""
    return 1.25 * wl.graph.V * (1 << k) * (D + 1) * 4 + 1e9


def save_arrays(d, wl):
    """The graph and group arrays as .npy files that worker processes map."""
    import numpy as np
    for nm, a in (("rowptr", wl.graph.rowptr), ("col", wl.graph.col), ("w", wl.graph.w),
                  ("gptr", wl.groups.ptr), ("gmem", wl.groups.mem)):
        path = os.path.join(d, f"arr_{nm}.npy")
        if not os.path.exists(path):
            np.save(path, a)


def lean_worker(d, D, query, out):
    """One restatement query in its own process: reads the mapped arrays,
    solves, checks the tree and writes {cost, seconds, pops} to `out`."""
    import numpy as np
    a = {nm: np.load(os.path.join(d, f"arr_{nm}.npy"), mmap_mode="r")
         for nm in ("rowptr", "col", "w", "gptr", "gmem")}
    g = dg.Graph(a["rowptr"], a["col"], a["w"])
    gr = dg.Groups(a["gptr"], a["gmem"])
    t0 = time.time()
    cost, edges, root, pops = oracle.hop_lean(g, gr, query, D)
    dt = time.time() - t0
    if cost < oracle.INF and oracle.validate(g, gr, query, edges, root, cost, D) != 0:
        raise SystemExit(f"restatement tree invalid for {query} D={D}")
    with open(out + ".tmp", "w") as f:
        json.dump({"cost": int(cost), "seconds": dt, "pops": int(pops)}, f)
    os.replace(out + ".tmp", out)


def run_jobs(jobs, procs, mem_budget, log):
    """Runs the jobs (dicts with argv, cwd, mem, done) with at most `procs`
    at once and the sum of their memory within the budget: the first listed
    job that fits starts, else the loop waits for one to end."""
    lock = threading.Condition()
    state = {"mem": 0.0, "run": 0}
    threads = []

    def work(job):
        t0 = time.time()
        try:
            subprocess.run(job["argv"], check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                           stdin=subprocess.DEVNULL, cwd=job["cwd"])
            job["wall"] = time.time() - t0
            job["done"](job)
        except Exception as e:  # a failed job leaves its cell unfinished
            log(f"{job['label']}: failed ({e})")
        finally:
            with lock:
                state["mem"] -= job["mem"]
                state["run"] -= 1
                lock.notify_all()

    todo = []
    for job in jobs:
        if job["mem"] > mem_budget:
            log(f"skip (needs {job['mem'] / 1e9:.0f} GB): {job['label']}")
        else:
            todo.append(job)
    while todo:
        with lock:
            def fits():
                return [j for j in todo if state["mem"] + j["mem"] <= mem_budget] if state["run"] < procs else []
            lock.wait_for(lambda: bool(fits()))
            job = fits()[0]
            todo.remove(job)
            state["mem"] += job["mem"]
            state["run"] += 1
        th = threading.Thread(target=work, args=(job,))
        th.start()
        threads.append(th)
    for th in threads:
        th.join()


def lean_jobs(name, wl, d, k, D, n, fx, save, wlock, log):
    """Jobs that pin the first n queries of cell (k, D) with the restatement,
    one process per query; queries an earlier restatement cell of the same
    inputs already pinned are kept, not rerun."""
    save_arrays(d, wl)
    queries = wl.queries
    idx = [i for i, (q, qd) in enumerate(queries) if len(q) == k and qd == D][:n]
    old = next((c for c in fx["cells"] if (c["k"], c["D"]) == (k, D) and c.get("program") == LEAN_PROGRAM), None)
    kept = {i: (c, t) for i, c, t in zip(old["idx"], old["costs"], old["oracle_time_s"])} if old else {}
    need = mem_bytes(wl, k, D) / 1e9
    cell = dict(k=k, D=D, idx=idx, queries=[queries[i][0].tolist() for i in idx],
                costs=[None] * len(idx), oracle_time_s=[None] * len(idx), program=LEAN_PROGRAM,
                reference_not_run=f"D-PrunedDP++ allocates its whole table up front: {need:.0f} GB "
                                  f"for k={k}, D={D} on {wl.graph.V:,} vertices")
    for j, i in enumerate(idx):
        if i in kept:
            cell["costs"][j], cell["oracle_time_s"][j] = kept[i]
    pending = {"n": sum(i not in kept for i in idx)}
    jobs = []
    for j, i in enumerate(idx):
        if i in kept:
            continue
        out = os.path.join(d, f"lean_{name}_k{k}_D{D}_{i}.json")
        argv = [sys.executable, os.path.abspath(__file__), "--lean-job", d, str(D),
                ",".join(str(int(x)) for x in queries[i][0]), out]

        def done(job, j=j, out=out):
            with open(out) as f:
                r = json.load(f)
            with wlock:
                cell["costs"][j] = r["cost"]
                cell["oracle_time_s"][j] = round(r["seconds"], 1)
                pending["n"] -= 1
                last = pending["n"] == 0
                if last:
                    fx["cells"] = [c for c in fx["cells"] if (c["k"], c["D"]) != (k, D)] + [cell]
            log(f"{job['label']}: {r['cost']} in {r['seconds']:.0f} s ({r['pops']} pops)")
            if last:
                save()

        jobs.append(dict(argv=argv, cwd=d, mem=lean_mem_bytes(wl, k, D), done=done,
                         label=f"{name} k={k} D={D} query {i} ({LEAN_PROGRAM})"))
    return jobs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("name", nargs="?", choices=sorted(SUBSETS))
    ap.add_argument("--procs", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    ap.add_argument("--mem-gb", type=float, default=48.0)
    ap.add_argument("--data-dir", default="", help="reuse a directory holding the written dataset")
    ap.add_argument("--restatement", action="store_true",
                    help="pin the cells the reference cannot run with oracle.hop_lean")
    ap.add_argument("--lean-job", nargs=4, metavar=("DIR", "D", "QUERY", "OUT"), help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.lean_job:
        d, D, q, out = args.lean_job
        lean_worker(d, int(D), [int(x) for x in q.split(",")], out)
        return
    if not args.name:
        ap.error("name the dataset (c3 or c4)")
    name = args.name
    out_path = os.path.join(HERE, f"{FIXTURE_FILE.get(name, name)}.json")
    wl, spec = workload(name)
    queries = wl.queries
    fx = dict(name=name, spec=spec, checksum=mg.checksum(wl.graph, wl.groups), cells=[],
              generated_by="tests/golden/make_golden_large.py (reference PrunedDP++ / D-PrunedDP++ built "
                           "from source by oracle/Makefile, one single-threaded process per query range)")
    if os.path.exists(out_path):  # resume: keep the finished cells of the same inputs
        with open(out_path) as f:
            old = json.load(f)
        if old.get("checksum") == fx["checksum"]:
            fx["cells"] = [c for c in old.get("cells", []) if c.get("costs") or c.get("not_pinned")]
    # A cell smaller than its subset is extended: its pinned queries are kept
    # and only the missing ones run.  With --restatement the not-pinned cells
    # are the ones to redo; each keeps its record until its replacement is
    # finished.
    lean = LEAN_SUBSETS.get(name, {})

    def finished(c):
        key = (c["k"], c["D"])
        if c.get("program") == LEAN_PROGRAM:
            return not args.restatement or len(c["idx"]) >= lean.get(key, 0)
        if c.get("costs"):
            avail = sum(len(q) == c["k"] and qd == c["D"] for q, qd in queries)
            return len(c["idx"]) >= min(SUBSETS[name].get(key, 0), avail)
        return not args.restatement
    done_cells = {(c["k"], c["D"]) for c in fx["cells"] if finished(c)}
    wlock = threading.Lock()

    def log(msg):
        print(time.strftime("%H:%M:%S"), msg, flush=True)

    def save():
        with wlock:
            fx["cells"].sort(key=lambda c: (c["D"] >= 0, c["k"], c["D"]))
            with open(out_path + ".tmp", "w") as f:
                json.dump(fx, f, indent=1)
            os.replace(out_path + ".tmp", out_path)

    d = args.data_dir or tempfile.mkdtemp(prefix=f"gstgold_{name}_")
    os.makedirs(os.path.join(d, "result"), exist_ok=True)
    log(f"work directory {d}")

    def ensure_dataset():  # the reference programs' text input files
        if not os.path.exists(os.path.join(d, name + ".in")):
            dg.write_dataset(d, name, dg.Workload(wl.graph, wl.groups, []), binary=False)

    jobs = []
    for (k, D), n in SUBSETS[name].items():
        if (k, D) in done_cells:
            continue
        idx = [i for i, (q, qd) in enumerate(queries) if len(q) == k and qd == D][:n]
        cell = dict(k=k, D=D, idx=idx, queries=[queries[i][0].tolist() for i in idx])
        if n == 0 and args.restatement and LEAN_SUBSETS.get(name, {}).get((k, D)):
            jobs += lean_jobs(name, wl, d, k, D, LEAN_SUBSETS[name][(k, D)], fx, save, wlock, log)
            continue
        if n == 0:
            if any(len(q) == k and qd == D for q, qd in queries):
                need = mem_bytes(wl, k, D) / 1e9
                cell.update(idx=[], queries=[], costs=None, program=None,
                            not_pinned=f"D-PrunedDP++ allocates its whole table up front: {need:.0f} GB "
                                       f"for k={k}, D={D} on {wl.graph.V:,} vertices")
                fx["cells"].append(cell)
            continue
        if not idx:
            continue
        prog = "PrunedDP++" if D < 0 else "D-PrunedDP++"
        old = next((c for c in fx["cells"] if (c["k"], c["D"]) == (k, D) and c.get("program") == prog
                    and c.get("costs")), None)
        kept = {i: (c, t) for i, c, t in zip(old["idx"], old["costs"], old["ref_time_s"])} if old else {}
        cell.update(costs=[kept[i][0] if i in kept else None for i in idx],
                    ref_time_s=[kept[i][1] if i in kept else None for i in idx], program=prog)
        todo = [i for i in idx if i not in kept]  # the queries this run solves, in cell order
        pos = {i: j for j, i in enumerate(idx)}
        if not todo:
            continue
        ensure_dataset()
        # a data name per cell (and per extension): symlinks to the shared
        # graph and groups, the queries to solve as <data><k>.csv
        data = f"{name}_k{k}_" + ("plain" if D < 0 else f"D{D}") + (f"_from{len(kept)}" if kept else "")
        for ext in (".in", ".g"):
            dst = os.path.join(d, data + ext)
            if not os.path.exists(dst):
                os.symlink(os.path.join(d, name + ext), dst)
        dg.write_queries(os.path.join(d, f"{data}{k}.csv"), [queries[i] for i in todo])
        per = PLAIN_PER_JOB if D < 0 else 1
        pending = {"n": 0}
        for a in range(0, len(todo), per):
            b = min(a + per, len(todo)) - 1
            argv = [oracle.ref_binary(prog), "1" if D < 0 else "2", d + "/", data, str(k)]
            argv += ([str(D)] if D >= 0 else []) + [str(a), str(b)]
            tag = "CPU_nonHop" if D < 0 else "CPU_Hop"
            csv = os.path.join(d, "result", f"exp_{tag}_{data}_T{k}_" + (f"D{D}_" if D >= 0 else "") + f"{a}-{b}.csv")
            pending["n"] += 1

            def done(job, cell=cell, a=a, csv=csv, pending=pending, todo=todo, pos=pos, k=k, D=D):
                with open(csv) as f:
                    next(f)
                    rows = [ln.strip().split(",") for ln in f if ln.strip()]
                with wlock:
                    for j, r in enumerate(rows):
                        cell["costs"][pos[todo[a + j]]] = int(r[3])
                        cell["ref_time_s"][pos[todo[a + j]]] = float(r[2])
                    pending["n"] -= 1
                    last = pending["n"] == 0
                    if last:
                        fx["cells"] = [c for c in fx["cells"] if (c["k"], c["D"]) != (k, D)] + [cell]
                log(f"{job['label']}: {[r[3] for r in rows]} in {job['wall']:.0f} s")
                if last:
                    save()

            jobs.append(dict(argv=argv, cwd=d, mem=mem_bytes(wl, k, D), done=done,
                             label=f"{name} k={k} D={D} queries {[todo[x] for x in range(a, b + 1)]}"))
    jobs.sort(key=lambda j: -j["mem"])  # largest tables (the longest queries) first
    save()
    log(f"{len(jobs)} jobs, {args.procs} processes, {args.mem_gb} GB")
    run_jobs(jobs, args.procs, args.mem_gb * 1e9, log)
    save()
    log("done")


if __name__ == "__main__":
    main()
