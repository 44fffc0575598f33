"""Benchmark: GST queries/s on one B200 (or N replicas), exact costs.

A "step" is one batch of queries solved by the engine over the resident
graph.  The default workload is C4, the configuration the headline metric is
stated on: BA V=4,000,000 m=9 + spanning path, w U[1,100], 20,000 groups
Geom(12) in [2,1000], 300 queries with k uniform in {3,5,7}, half of them
diameter-bounded (D uniform in [2,5]).  Seeded synthetic data stands in for
the reference's external social graphs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c4|c2|c1]
                    [--impl ours|reference]
    python bench.py --workload c5 [--rates 50,200,1000] [--serve-queries 10000]

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events on the
engine's stream) whole-job queries/s with the graph resident in HBM; `e2e`
is the same metric through the C ABI with host buffers (query ids in, costs
and tree edges out) timed by the host clock around the call.
`single_query_qps` times the same engine one query per call on a sample of
every (k, plain / D-bounded) class and weights the classes as the batch
does; `batched_over_single` is the ratio.  `parity` compares the batch's
costs with the reference costs committed under tests/golden/ for this
workload.  `roofline` is the grow kernel's algorithmic bytes per second
(events captured around each grow launch) against the measured HBM copy
bandwidth.  `cpu_baseline` times the reference's own PrunedDP++ (built from
source into oracle/_ref) on a bounded sample of the workload's plain
queries, per query from its own progress lines (graph load excluded), and
scales it to the host cores.  --impl reference times that reference CPU
path alone.  --workload c5 is the serving loop: Poisson arrivals on the C4
graph, one JSON line per arrival rate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu4gst-1_b200"))
sys.path.insert(0, ROOT)

from gst_b200.clocks import ClockSampler  # noqa: E402

METRIC = "GST queries/sec (k=3/5/7) batched vs 1-query GPU at exact cost; p50/p99; HBM %"

WORKLOADS = {
    "c1": "C1: BA V=10,000 m=5, w U[1,100]; 500 groups U[2,20]; 50 queries k=3",
    "c2": "C2: BA V=170,000 m=20 + spanning path, w U[1,100]; 3,000 groups Geom(8) in [2,200]; "
          "300 queries k=5",
    "c4": "C4: BA V=4,000,000 m=9 + spanning path, w U[1,100]; 20,000 groups Geom(12) in [2,1000]; "
          "300 queries k in {3,5,7}, half D=inf, half D in [2,5]",
}


def make_workload(name: str, rank: int):
    from gst_b200 import datagen as dg
    seed = 1 + 1000 * rank  # weak scaling: every rank solves its own query set
    if name == "c1":
        wl = dg.config_c1(1)
        wl.queries = dg.make_queries(wl.groups.n, 50, 3, seed + 200)
    elif name == "c2":
        wl = dg.config_c2(1, n_queries=1)
        wl.queries = dg.make_queries(wl.groups.n, 300, 5, seed + 200)
    elif name == "c4":
        wl = dg.config_c4(1, n_queries=1)
        wl.queries = dg.make_queries(wl.groups.n, 300, [3, 5, 7], seed + 200,
                                     D=lambda r: -1 if r.random() < 0.5 else int(r.integers(2, 6)))
    else:
        raise SystemExit(f"unknown workload {name}")
    return wl


def c5_queries(n_groups: int, n: int):
    """The serving mix on the C4 graph and groups: k in {3,5,7} with
    probabilities {0.5,0.3,0.2}; D unbounded with probability 0.5, else
    uniform in [2,5]; seed 7."""
    from gst_b200 import datagen as dg
    return dg.make_queries(n_groups, n, ([3, 5, 7], [0.5, 0.3, 0.2]), 7,
                           D=lambda r: -1 if r.random() < 0.5 else int(r.integers(2, 6)))


def query_class(q, D) -> str:
    return f"k{len(q)}_" + ("plain" if D < 0 else "D")


def arrays_checksum(g, gr) -> str:
    """sha256 prefix of the generated graph and group arrays (the recipe the
    committed fixtures under tests/golden/ carry)."""
    import hashlib
    import numpy as np
    h = hashlib.sha256()
    for a in (g.rowptr, g.col, g.w, gr.ptr, gr.mem):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def fixture_parity(name: str, wl, costs) -> dict | None:
    """Compares the batch's costs with the reference costs committed in
    tests/golden/<name>.json, or <name>_batch.json (the queries there are this
    workload's own, by index).  Raises if one differs."""
    fx = None
    for fn in (f"{name}.json", f"{name}_batch.json"):
        path = os.path.join(ROOT, "tests", "golden", fn)
        if not os.path.exists(path):
            continue
        with open(path) as f:
            cand = json.load(f)
        if "cells" in cand and cand.get("checksum") == arrays_checksum(wl.graph, wl.groups):
            fx = cand
            break
    if fx is None:
        return None
    n = 0
    by_program = {}
    for c in fx["cells"]:
        if not c.get("costs"):
            continue
        prog = c.get("program") or "reference"
        for i, want in zip(c["idx"], c["costs"]):
            if want is None:
                continue
            assert costs[i] == want, f"query {i} (k={c['k']}, D={c['D']}): {costs[i]} != {prog} {want}"
            n += 1
            by_program[prog] = by_program.get(prog, 0) + 1
    return {"fixture": f"tests/golden/{fn}", "queries_checked": n, "equal": True,
            "by_program": by_program,
            "against": "reference PrunedDP++ / D-PrunedDP++ costs; oracle.hop_lean (the HOP_cpu "
                       "restatement) only on cells whose reference table does not fit in memory"}


def filter_queries(wl, args):
    """Optional sub-selection of a workload's queries (profiling small cases)."""
    qs = wl.queries
    if args.k > 0:
        qs = [(q, D) for q, D in qs if len(q) == args.k]
    if args.kind == "plain":
        qs = [(q, D) for q, D in qs if D < 0]
    elif args.kind == "hop":
        qs = [(q, D) for q, D in qs if D >= 0]
    if args.queries > 0:
        qs = qs[: args.queries]
    wl.queries = qs


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def random_read_ceiling(torch, device) -> dict:
    """Random 4-byte reads per second that a library gather reaches on this
    GPU: torch.take of 64 Mi uniformly random int32 from a 4 GiB array (each
    read costs at least a 32-byte sector).  It is the access pattern of the
    grow kernel's target reads, so it bounds the grow better than the copy
    bandwidth does."""
    x = torch.empty(1 << 30, dtype=torch.int32, device=device)
    x.fill_(1)
    idx = torch.randint(0, 1 << 30, (64 << 20,), dtype=torch.int64, device=device)
    out = torch.empty(64 << 20, dtype=torch.int32, device=device)
    best = None
    for _ in range(4):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        torch.take(x, idx, out=out)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    del x, idx, out
    torch.cuda.empty_cache()
    return {"reads_per_s": (64 << 20) / (best / 1e3), "sector_gbs": (64 << 20) * 32 / (best / 1e3) / 1e9,
            "how": "torch.take: 64 Mi random int32 reads from a 4 GiB array, best of 4"}


def flush_l2(torch, buf):
    buf.fill_(1.0)  # 256 MB write, larger than the 126 MB L2
    torch.cuda.synchronize()


def grow_bytes(stats_sum):
    """Algorithmic bytes of the grow kernel: 16 per expanded state (own cost 4,
    CSR offsets 8, frontier entry 4), 12 per edge relaxation (neighbour 4,
    weight 4, target read 4) and 4 per successful update (write)."""
    return 16 * stats_sum["frontier"] + 12 * stats_sum["relax"] + 4 * stats_sum["improve"]


def write_dataset_files(name: str, out_dir: str) -> dict:
    """Writes the workload's graph and groups in the reference's text formats
    and its plain queries by k, from a child process, so that the process
    timing the reference never maps this project's libraries.  Returns the
    plain queries as {k: [[ids], ...]} in workload order."""
    meta = os.path.join(out_dir, "meta.json")
    if not os.path.exists(meta):
        subprocess.run([sys.executable, os.path.abspath(__file__), "--write-dataset", out_dir,
                        "--workload", name], check=True, stdin=subprocess.DEVNULL)
    with open(meta) as f:
        return {int(k): v for k, v in json.load(f).items()}


def _write_dataset_main(name: str, out_dir: str) -> None:
    from gst_b200 import datagen as dg
    wl = make_workload(name, 0)
    dg.write_dataset(out_dir, name, dg.Workload(wl.graph, wl.groups, []), binary=False)
    byk = {}
    for q, D in wl.queries:
        if D < 0:
            byk.setdefault(len(q), []).append([int(x) for x in q])
    for k, qs in byk.items():
        with open(os.path.join(out_dir, f"{name}{k}.csv"), "w") as f:
            for q in qs:
                f.write(" ".join(map(str, q)) + "\n")
    with open(os.path.join(out_dir, "meta.json.tmp"), "w") as f:
        json.dump(byk, f)
    os.replace(os.path.join(out_dir, "meta.json.tmp"), os.path.join(out_dir, "meta.json"))


def run_ref_timed(exe: str, d: str, name: str, k: int, a: int, b: int, budget_s: float):
    """Runs the reference PrunedDP++ on queries a..b of <name><k>.csv and
    times each query from its own progress lines: "<data> iteration i" is
    printed when query i starts and a line of dashes when its solve and
    feasibility check are done (code/PrunedDP++/include/exp_CPU_nonHop.h:90-127),
    so the graph load and the process's teardown are excluded and each
    query's own preprocessing is counted.  The process is stopped budget_s
    seconds after its first query started.  Returns (the finished queries'
    times, the time the unfinished query had run when it was stopped, or
    None): the latter is a lower bound on that query's time."""
    p = subprocess.Popen([exe, "1", d + "/", name, str(k), str(a), str(b)], stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, text=True)
    times = []
    t_start = None
    timer = None

    def stop():
        if p.poll() is None:
            p.kill()

    for line in p.stdout:
        if " iteration " in line:
            t_start = time.perf_counter()
            if timer is None:
                timer = threading.Timer(budget_s, stop)
                timer.start()
        elif line.startswith("-----") and t_start is not None:
            times.append(time.perf_counter() - t_start)
            t_start = None
    p.wait()
    if timer is not None:
        timer.cancel()
    cut = time.perf_counter() - t_start if t_start is not None else None
    return times, cut


def sample_positions(n: int, per_k: int) -> list:
    """per_k positions spread evenly over a class of n queries (0, n/per_k,
    2n/per_k, ...): query times within a class spread over two orders of
    magnitude, so the first queries alone are no fair sample."""
    m = min(per_k, n)
    return [j * n // m for j in range(m)]


def cpu_reference_sample(name: str, per_k: int, budget_s: float = 300):
    """The reference PrunedDP++ (oracle/_ref) on per_k plain queries of each
    k of the workload, spread evenly over the class, one single-threaded
    process per query, all at once, each stopped budget_s seconds after its
    query started.  Returns per-class mean seconds per query (a stopped query
    counts with the time it had run: a lower bound) and what ran."""
    import oracle
    exe = oracle.ref_binary("PrunedDP++")
    if not os.path.exists(exe):
        return None
    d = os.path.join(tempfile.gettempdir(), f"gstbench_{name}")
    os.makedirs(os.path.join(d, "result"), exist_ok=True)
    byk = write_dataset_files(name, d)
    jobs = [(k, i) for k in sorted(byk) for i in sample_positions(len(byk[k]), per_k)]
    out = [None] * len(jobs)

    def one(j):
        k, i = jobs[j]
        out[j] = run_ref_timed(exe, d, name, k, i, i, budget_s)

    ths = [threading.Thread(target=one, args=(j,)) for j in range(len(jobs))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    per, stopped = {}, 0
    for (k, i), (ts, cut) in zip(jobs, out):
        if ts:
            per.setdefault(k, []).append(ts[0])
        elif cut is not None:
            per.setdefault(k, []).append(cut)
            stopped += 1
    return {"per_k_s": {k: statistics.mean(v) for k, v in per.items()}, "queries": len(jobs),
            "per_k": per_k, "stopped": stopped, "budget_s": budget_s,
            "positions": {k: sample_positions(len(byk[k]), per_k) for k in sorted(byk)}}


def cpu_mix_qps(per_k_s: dict, queries, cores: int):
    """Queries/s of `cores` single-threaded reference processes on the
    plain-query mix of the workload (each class weighted by its count)."""
    plain = [len(q) for q, D in queries if D < 0 and len(q) in per_k_s]
    if not plain:
        return None
    mean_s = sum(per_k_s[k] for k in plain) / len(plain)
    return cores / mean_s


def reference_gpu_sample(wl, name: str, n: int, timeout: float = 900):
    """Runs the reference GPU program TrimCDP (built for sm_100a into
    oracle/_ref) on the first n plain queries of the workload, one query after
    another as the reference does.  Returns its wall time (incl. its graph
    load), its own Relax-loop times (its `rt` column) and its costs.  A GPU
    comparator beside the CPU baseline, not the CPU baseline."""
    import oracle
    from gst_b200 import datagen as dg
    exe = oracle.ref_binary("TrimCDP")
    if not os.path.exists(exe):
        return None
    d = tempfile.mkdtemp(prefix="gstrefgpu_")
    plain = [(q, D) for q, D in wl.queries if D < 0]
    k = sorted({len(q) for q, _ in plain})[0]
    qs = [(q, D) for q, D in plain if len(q) == k][:n]
    dg.write_dataset(d, name, dg.Workload(wl.graph, wl.groups, []), binary=False)
    dg.write_queries(os.path.join(d, f"{name}{k}.csv"), qs)
    t0 = time.time()
    subprocess.run([exe, "2", d + "/", name, str(k), "0", str(len(qs) - 1)], check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL, timeout=timeout)
    wall = time.time() - t0
    rt, cost = [], []
    with open(os.path.join(d, "result", f"exp_GPU1_nonHop_{name}_T{k}_0-{len(qs) - 1}.csv")) as f:
        next(f)
        for line in f:
            if line.strip():
                p = line.split(",")
                rt.append(float(p[2]))
                cost.append(int(p[3]))
    return {"queries": len(qs), "k": k, "wall_s": wall, "relax_loop_s_median": statistics.median(rt),
            "relax_loop_s_total": sum(rt), "costs": cost}


def run_serving(args):
    """C5: the serving loop (continuous batching) on the C4 graph and groups
    under Poisson arrivals, one JSON line per rate.  Latency runs from a
    query's submission to its result being ready on the host (measured by
    the engine); every served cost must equal the engine's batch answer for
    the same query, and the C4 batch is checked against the reference costs
    of the C4 fixture."""
    import numpy as np
    import gst_b200
    wl = make_workload("c4", 0)
    queries = c5_queries(wl.groups.n, args.serve_queries)
    eng = gst_b200.Engine(device=0, arena_bytes=int(args.arena_gb * (1 << 30)),
                          max_slots=args.max_slots, rounds_per_poll=args.rounds_per_poll)
    eng.load_graph(wl.graph.rowptr, wl.graph.col, wl.graph.w)
    eng.load_groups(wl.groups.ptr, wl.groups.mem)
    c4_costs = [r.cost for r in eng.solve_batch([q for q, _ in wl.queries], [D for _, D in wl.queries])]
    parity = fixture_parity("c4", wl, c4_costs)
    t0 = time.perf_counter()
    alone = [r.cost for r in eng.solve_batch([q for q, _ in queries], [D for _, D in queries])]
    batch_s = time.perf_counter() - t0
    mix = {}
    for q, D in queries:
        mix[query_class(q, D)] = mix.get(query_class(q, D), 0) + 1
    for rate in args.rates:
        gaps = np.random.default_rng(7).exponential(1.0 / rate, size=len(queries))
        tickets = []
        sampler = ClockSampler(0)
        sampler.start()
        with eng.server() as srv:
            t0 = time.perf_counter()
            t_next = t0
            for i, (q, D) in enumerate(queries):
                t_next += gaps[i]
                while True:
                    dt = t_next - time.perf_counter()
                    if dt <= 0:
                        break
                    time.sleep(min(dt, 0.001))
                tickets.append(srv.submit(q, D))
            res = [srv.wait(t) for t in tickets]
            span = time.perf_counter() - t0
        clocks = sampler.stop()
        lat = np.array([r.stats["latency_ms"] for r in res])
        qwait = np.array([r.stats["queue_ms"] for r in res])
        got = [r.cost for r in res]
        bad = sum(1 for a, b in zip(got, alone) if a != b)
        assert all(r.status == 0 for r in res), "a served query failed"
        print(json.dumps({
            "mode": "serving", "workload": "C5: the C4 graph and groups; Poisson arrivals, seed 7; "
            "k in {3,5,7} w.p. {.5,.3,.2}; D=inf w.p. .5, else U[2,5]",
            "arrival_rate_qps": rate, "queries": len(queries), "mix": mix, "served_qps": len(queries) / span,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                           "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "admission_wait_ms": {"p50": float(np.percentile(qwait, 50)), "p99": float(np.percentile(qwait, 99))},
            "results_equal_batch": bad == 0, "results_differing": bad,
            "batch_same_queries_qps": len(queries) / batch_s,
            "parity_c4": parity, "clocks": clocks}), flush=True)
        assert bad == 0, f"{bad} served costs differ from the batch answer"
    eng.close()


def run_reference_arm(args):
    """The reference's own CPU path (PrunedDP++ from oracle/_ref) on the host
    cores, on this workload's plain queries.  One single-threaded process per
    core; process p runs queries of class k = ks[p % len(ks)] one after
    another (warm-up queries first), timed from the reference's own progress
    lines (graph load excluded) and stopped after a time budget.  value =
    cores / the mean time per query of the plain-query mix (each class
    weighted by its share of the workload's plain queries): the throughput of
    the host cores kept busy on that mix."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    exe = oracle.ref_binary("PrunedDP++")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/PrunedDP++ is not built"}), flush=True)
        return
    procs = max(1, min(os.cpu_count() or 1, 32))
    d = os.path.join(tempfile.gettempdir(), f"gstbench_{args.workload}")
    os.makedirs(os.path.join(d, "result"), exist_ok=True)
    byk = write_dataset_files(args.workload, d)
    ks = sorted(byk)
    per = args.warmup + args.steps
    got = {}

    def one(p):
        k = ks[p % len(ks)]
        n = len(byk[k])
        a = ((p // len(ks)) * per) % n
        b = min(n, a + per) - 1
        got[p] = (k, run_ref_timed(exe, d, args.workload, k, a, b, budget_s=args.ref_budget))

    ths = [threading.Thread(target=one, args=(p,)) for p in range(procs)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    # the graph load of each process is its warm-up; a query still running at
    # the budget counts with the time it had run (a lower bound on its time)
    per_k, stopped = {}, 0
    for k, (ts, cut) in got.values():
        per_k.setdefault(k, []).extend(ts)
        if not ts and cut is not None:
            per_k[k].append(cut)
            stopped += 1
    mean_k = {k: statistics.mean(v) for k, v in per_k.items() if v}
    weights = {k: len(v) for k, v in byk.items() if k in mean_k}
    t_mix = sum(weights[k] * mean_k[k] for k in weights) / sum(weights.values())
    v = procs / t_mix
    nq = sum(len(v) for v in per_k.values())
    sample = (f"{nq} timed plain queries of the {args.workload.upper()} workload on {procs} single-threaded "
              f"PrunedDP++ processes (process p runs k = {ks}[p mod {len(ks)}], stopped {args.ref_budget:.0f} s "
              f"after its first query; {stopped} stopped in their first query count with the time they had "
              f"run); per-query time from the reference's progress lines (graph load excluded); "
              f"value = {procs} / the plain-query mix's mean s per query; mean s by k: "
              + ", ".join(f"k={k}: {mean_k[k]:.2f}" for k in sorted(mean_k)))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_mix,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": {"workload": WORKLOADS[args.workload]},
        "cpu_baseline": {"value": v, "unit": "queries/s", "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOADS) + ["c5"],
                    help="c5: the serving loop on the C4 graph")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--single-per-class", type=int, default=10,
                    help="queries of each (k, plain / D-bounded) class timed one per call")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--queries", type=int, default=0, help="queries per step (0: the workload's count)")
    ap.add_argument("--arena-gb", type=float, default=0.0, help="device arena size (0: 85%% of free memory)")
    ap.add_argument("--max-slots", type=int, default=0, help="queries resident at once (0: engine default)")
    ap.add_argument("--rounds-per-poll", type=int, default=0)
    ap.add_argument("--bucket-shift", type=int, default=0, help="cost-bucket width = best >> shift (0: engine default)")
    ap.add_argument("--k", type=int, default=0, help="keep only queries with this many groups (0: all)")
    ap.add_argument("--kind", default="all", choices=["all", "plain", "hop"],
                    help="keep only plain (D unbounded) or diameter-bounded queries")
    ap.add_argument("--ref-gpu", type=int, default=0,
                    help="also run the reference GPU TrimCDP on this many plain queries (comparator)")
    ap.add_argument("--rates", default="50,200,1000", help="c5: Poisson arrival rates, queries/s")
    ap.add_argument("--serve-queries", type=int, default=10000, help="c5: queries per rate")
    ap.add_argument("--ref-budget", type=float, default=360.0,
                    help="reference arm: seconds each reference process runs after its first query")
    ap.add_argument("--cpu-per-k", type=int, default=3,
                    help="cpu_baseline: plain queries per k, spread evenly over the class")
    ap.add_argument("--cpu-budget", type=float, default=300.0,
                    help="cpu_baseline: seconds a reference process may run its query")
    ap.add_argument("--tuning", default="auto",
                    help="engine parameter file (auto: gpu4gst-1_b200/tuning/<workload>.json if present; none)")
    ap.add_argument("--write-dataset", default="", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.write_dataset:
        return _write_dataset_main(args.workload, args.write_dataset)
    args.warmup = max(args.warmup, 3)
    args.rates = [float(x) for x in args.rates.split(",") if x]
    if args.workload == "c5":
        return run_serving(args)
    if args.impl == "reference":
        return run_reference_arm(args)

    import numpy as np
    import torch
    import gst_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    unfiltered = not (args.k or args.kind != "all" or args.queries)
    # the reference CPU sample runs on host cores while the GPU steps run
    cpu_sample = {}
    cpu_thread = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and unfiltered:
        def _cpu():
            cpu_sample["r"] = cpu_reference_sample(args.workload, per_k=args.cpu_per_k, budget_s=args.cpu_budget)
        cpu_thread = threading.Thread(target=_cpu, daemon=True)
        cpu_thread.start()
    wl = make_workload(args.workload, rank)
    filter_queries(wl, args)
    queries = [q for q, _ in wl.queries]
    Ds = [D for _, D in wl.queries]
    ceiling = random_read_ceiling(torch, f"cuda:{local}")  # before the engine takes its arena
    eng = gst_b200.Engine(device=local, profile=True, arena_bytes=int(args.arena_gb * (1 << 30)),
                          max_slots=args.max_slots, rounds_per_poll=args.rounds_per_poll,
                          bucket_shift=args.bucket_shift)
    eng.load_graph(wl.graph.rowptr, wl.graph.col, wl.graph.w)
    eng.load_groups(wl.groups.ptr, wl.groups.mem)
    tuning_file = None
    if args.tuning != "none":
        tuning_file = (os.path.join(ROOT, "gpu4gst-1_b200", "tuning", f"{args.workload}.json")
                       if args.tuning == "auto" else args.tuning)
        if os.path.exists(tuning_file):
            eng.load_tuning(tuning_file)
        else:
            tuning_file = None
    for key, v in (("rounds_per_poll", args.rounds_per_poll), ("max_slots", args.max_slots)):
        if v:  # explicit flags win over the parameter file
            eng.set_tuning({key: v})
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        res = eng.solve_batch(queries, Ds)
    assert all(r.status == 0 for r in res), "a warm-up query failed"

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    sampler = ClockSampler(local)
    sampler.start()
    dev_ms, wall_s, lat = [], [], []
    sums = {"frontier": 0, "relax": 0, "improve": 0, "merges": 0}
    grow_ms = merge_ms = 0.0
    grow_launches = launches = h2d = d2h = 0
    costs = None
    for _ in range(args.steps):
        flush_l2(torch, flush)
        barrier()
        t0 = time.perf_counter()
        res = eng.solve_batch(queries, Ds)
        wall_s.append(time.perf_counter() - t0)
        p = eng.profile()
        dev_ms.append(p["run_ms"])
        grow_ms += p["grow_ms"]
        merge_ms += p["merge_ms"]
        grow_launches += p["grow_launches"]
        launches += p["kernel_launches"]
        h2d += p["h2d_bytes"]
        d2h += p["d2h_bytes"]
        for r in res:
            for f in sums:
                sums[f] += r.stats[f]
            lat.append(r.stats["device_ms"])
        c = [r.cost for r in res]
        assert costs is None or c == costs, "costs changed between steps"
        costs = c
    barrier()
    clocks = sampler.stop()
    parity = fixture_parity(args.workload, wl, costs) if unfiltered else None

    # one-query-per-call form of the same engine (the "plain" GPU form): the
    # first queries of every (k, kind) class, weighted as the batch mixes them
    classes = {}
    for i, (q, D) in enumerate(zip(queries, Ds)):
        classes.setdefault(query_class(q, D), []).append(i)
    single = {}
    for cl, idx in sorted(classes.items()):
        ms = []
        for i in idx[: args.single_per_class]:
            r = eng.solve(queries[i], Ds[i])
            assert r.cost == costs[i], "one-query form disagrees with the batch"
            ms.append(eng.profile()["run_ms"])
        if ms:
            single[cl] = {"queries_in_batch": len(idx), "timed": len(ms), "mean_ms": statistics.mean(ms)}
    single_qps = None
    if single and all(cl in single for cl in classes):
        single_qps = len(queries) / (sum(v["queries_in_batch"] * v["mean_ms"] for v in single.values()) / 1e3)

    nq = len(queries)
    tot_dev = sum(dev_ms) / 1e3
    tot_wall = sum(wall_s)
    if dist is not None:
        t = torch.tensor([tot_dev, tot_wall], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_dev, tot_wall = float(t[0]), float(t[1])
    value = world * nq * args.steps / tot_dev
    e2e = world * nq * args.steps / tot_wall

    peak, peak_kind = peaks()
    grow_reads = sums["relax"] / (grow_ms / 1e3) if grow_ms > 0 else None
    gb = grow_bytes(sums)
    achieved = gb / (grow_ms / 1e3) / 1e9 if grow_ms > 0 else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"grow_{args.workload}_traffic.json")
    if os.path.exists(tp) and unfiltered:
        with open(tp) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")

    out = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded BA power-law graphs standing in for the reference's external datasets)",
        "config": {"workload": WORKLOADS[args.workload], "queries_per_step_per_gpu": nq,
                   **({"query_filter": f"k={args.k or 'any'} kind={args.kind} first={args.queries or 'all'}"}
                      if not unfiltered else {}),
                   "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) before every step; "
                   "per-query DP tables (GBs per step) exceed L2",
                   "tuning": {"file": os.path.relpath(tuning_file, ROOT) if tuning_file else None,
                              "params": {k: v for k, v in eng.get_tuning().items()
                                         if k in ("grow_lanes", "rounds_per_poll", "max_slots", "overlap")}}},
        "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "single_query_qps": single_qps,
        "single_query_sample": {"per_class": single,
                                "how": f"first {args.single_per_class} queries of each (k, kind) class, one per "
                                       "call; classes weighted by their count in the batch"},
        "batched_over_single": (value / world) / single_qps if single_qps else None,
        "parity": parity,
        "latency_ms_in_batch": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                                "p99": float(np.percentile(lat, 99)),
                                "note": "admission to answer with the whole batch admitted at once"},
        "state_relaxations_per_s": world * sums["relax"] / tot_dev,
        "roofline": {"kernel": "k_grow", "bound": "hbm", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": traffic,
                     "algorithmic_bytes_per_launch": gb / max(grow_launches, 1),
                     "avg_launch_ms": grow_ms / max(grow_launches, 1),
                     "grow_share_of_device_time": grow_ms / (tot_dev * 1e3) if tot_dev else None,
                     "merge_ms_per_step": merge_ms / args.steps,
                     "merge_share_of_device_time": merge_ms / (tot_dev * 1e3) if tot_dev else None,
                     # the grow's target reads are random 4-byte reads: their
                     # rate against a library random gather on the same GPU
                     "random_reads": {"grow_target_reads_per_s": grow_reads,
                                      "ceiling": ceiling,
                                      "frac": grow_reads / ceiling["reads_per_s"] if grow_reads else None}},
        "clocks": clocks,
    }
    if cpu_thread is not None:
        cpu_thread.join()
        cores = max(1, min(os.cpu_count() or 1, 32))
        smp = cpu_sample.get("r")
        if smp is not None:
            qps = cpu_mix_qps(smp["per_k_s"], wl.queries, cores)
            out["cpu_baseline"] = {
                "value": qps, "unit": "queries/s", "cores": cores, "kind": "reference",
                "sample": f"{smp['per_k']} plain queries of each k of this workload (spread evenly over "
                          f"the class: positions {smp['positions']}), one "
                          f"single-threaded PrunedDP++ process each ({smp['queries']} at once, on host cores "
                          f"while the GPU steps ran); per-query time from the reference's progress lines "
                          f"(graph load excluded); {smp['stopped']} queries still running after "
                          f"{smp['budget_s']:.0f} s count with the time they had run (a lower bound); value = "
                          f"{cores} cores / the plain-query mix's mean time per query; mean s per query "
                          "by k: " + ", ".join(f"k={k}: {t:.2f}" for k, t in sorted(smp["per_k_s"].items()))}
    if rank == 0 and args.ref_gpu > 0:
        eng.close()
        torch.cuda.empty_cache()
        ref = reference_gpu_sample(wl, args.workload, args.ref_gpu)
        if ref is not None:
            plain = [i for i, (q, D) in enumerate(wl.queries) if D < 0 and len(q) == ref["k"]]
            ref["costs_equal_ours"] = ref.pop("costs") == [costs[i] for i in plain[: ref["queries"]]]
            ref["queries_per_s_relax_loop_only"] = ref["queries"] / ref["relax_loop_s_total"]
            out["reference_gpu_trimcdp"] = ref
    if rank == 0:
        print(json.dumps(out), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
