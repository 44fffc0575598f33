"""Benchmark: GST queries/s on one B200 (or N replicas), exact costs.

A "step" is one batch of queries solved by the engine over the resident
graph (default workload C2: BA V=170,000 m=20 + spanning path, w U[1,100],
3,000 groups Geom(8) in [2,200], 300 queries of k=5; seeded synthetic data
standing in for the reference's external social graphs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c4|c1]
                    [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events on the
engine's stream) whole-job queries/s with the graph resident in HBM; `e2e`
is the same metric through the C ABI with host buffers (query ids in, costs
and tree edges out) timed by the host clock around the call.  `roofline` is
the grow kernel's algorithmic bytes per second (events captured around each
grow launch) against the measured HBM copy bandwidth.  `cpu_baseline` runs
the reference's own PrunedDP++ (built from source into oracle/_ref) on a
bounded sample of the same workload, one process per core as the reference's
scripts do.  --impl reference times that reference CPU path alone.
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


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(torch, buf):
    buf.fill_(1.0)  # 256 MB write, larger than the 126 MB L2
    torch.cuda.synchronize()


def grow_bytes(stats_sum):
    """Algorithmic bytes of the grow kernel: 16 per expanded state (own cost 4,
    CSR offsets 8, frontier entry 4), 12 per edge relaxation (neighbour 4,
    weight 4, target read 4) and 4 per successful update (write)."""
    return 16 * stats_sum["frontier"] + 12 * stats_sum["relax"] + 4 * stats_sum["improve"]


def cpu_reference_sample(wl, name: str, n_queries: int, procs: int, timeout: float = 600):
    """Runs the reference PrunedDP++ binary (oracle/_ref) on the first
    n_queries queries of the workload, `procs` processes on disjoint query
    ranges.  Returns (queries/s by wall clock, per-query reference CSV times, kind)."""
    import oracle
    from gst_b200 import datagen as dg
    exe = oracle.ref_binary("PrunedDP++")
    d = tempfile.mkdtemp(prefix="gstbench_")
    plain = [(q, D) for q, D in wl.queries if D < 0]
    ks = sorted({len(q) for q, _ in plain})
    k = ks[0]
    qs = [(q, D) for q, D in plain if len(q) == k][:n_queries]
    dg.write_dataset(d, name, dg.Workload(wl.graph, wl.groups, []), binary=False)
    dg.write_queries(os.path.join(d, f"{name}{k}.csv"), qs)
    per = max(1, (len(qs) + procs - 1) // procs)
    ranges = [(s, min(s + per, len(qs)) - 1) for s in range(0, len(qs), per)]
    if os.path.exists(exe):
        kind = "reference"
        t0 = time.time()
        ps = [subprocess.Popen([exe, "1", d + "/", name, str(k), str(a), str(b)], stdout=subprocess.DEVNULL,
                               stderr=subprocess.DEVNULL, stdin=subprocess.DEVNULL) for a, b in ranges]
        for p in ps:
            p.wait(timeout=timeout)
        wall = time.time() - t0
        times = []
        try:
            for a, b in ranges:
                fn = os.path.join(d, "result", f"exp_CPU_nonHop_{name}_T{k}_{a}-{b}.csv")
                with open(fn) as f:
                    next(f)
                    for line in f:
                        if line.strip():
                            times.append(float(line.split(",")[2]))
        except OSError:
            pass
        return len(qs) / wall, times, kind, len(ranges), len(qs), k
    # no reference build on this box: the oracle port, one process per range
    import multiprocessing as mp
    kind = "port"
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(len(ranges)) as pool:
        pool.starmap(_port_range, [(wl, [q for q, _ in qs[a:b + 1]]) for a, b in ranges])
    wall = time.time() - t0
    return len(qs) / wall, [], kind, len(ranges), len(qs), k


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
    """Poisson arrivals at --serve queries/s through the engine's serving loop
    (continuous batching); reports per-query latency from submit to result and
    the sustained throughput."""
    import numpy as np
    import gst_b200
    wl = make_workload(args.workload, 0)
    filter_queries(wl, args)
    eng = gst_b200.Engine(device=0, arena_bytes=int(args.arena_gb * (1 << 30)))
    eng.load_graph(wl.graph.rowptr, wl.graph.col, wl.graph.w)
    eng.load_groups(wl.groups.ptr, wl.groups.mem)
    alone = eng.solve_batch([q for q, _ in wl.queries], [D for _, D in wl.queries])
    rng = np.random.default_rng(7)
    gaps = rng.exponential(1.0 / args.serve, size=len(wl.queries))
    lat = [None] * len(wl.queries)
    got = [None] * len(wl.queries)
    with eng.server() as srv:
        def waiter(i, ticket, t_sub):  # one waiter per request: latency = submit -> result
            r = srv.wait(ticket)
            lat[i] = time.perf_counter() - t_sub
            got[i] = r.cost

        ths = []
        t0 = time.perf_counter()
        t_next = t0
        for i, (q, D) in enumerate(wl.queries):
            t_next += gaps[i]
            while time.perf_counter() < t_next:
                time.sleep(0.0002)
            t_sub = time.perf_counter()
            th = threading.Thread(target=waiter, args=(i, srv.submit(q, D), t_sub))
            th.start()
            ths.append(th)
        for th in ths:
            th.join()
        span = time.perf_counter() - t0
    eng.close()
    ms = np.array(lat) * 1e3
    print(json.dumps({
        "mode": "serving", "workload": WORKLOADS[args.workload], "arrival_rate_qps": args.serve,
        "queries": len(wl.queries), "served_qps": len(wl.queries) / span,
        "latency_ms": {"p50": float(np.percentile(ms, 50)), "p90": float(np.percentile(ms, 90)),
                       "p99": float(np.percentile(ms, 99)), "max": float(ms.max())},
        "results_equal_alone": got == [r.cost for r in alone]}), flush=True)


def _port_range(wl, queries):
    import oracle
    for q in queries:
        oracle.prunedpp(wl.graph, wl.groups, q)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = make_workload(args.workload, 0)
    procs = max(1, min(os.cpu_count() or 1, 32))
    vals = []
    info = None
    for step in range(args.warmup + args.steps):
        qps, times, kind, nproc, nq, k = cpu_reference_sample(wl, args.workload, procs, procs)
        if step >= args.warmup:
            vals.append(qps)
        info = (kind, nproc, nq, k)
    kind, nproc, nq, k = info
    v = statistics.mean(vals) if vals else None
    sample = (f"{nq} queries (k={k}) of the {args.workload.upper()} workload per step, one "
              f"single-threaded PrunedDP++ process per query range, {nproc} processes")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]},
        "cpu_baseline": {"value": v, "unit": "queries/s", "cores": nproc, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--single", type=int, default=30, help="queries timed one per call")
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
    ap.add_argument("--serve", type=float, default=0.0,
                    help="serving mode: Poisson arrivals at this many queries/s (prints its own line)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.serve > 0:
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

    # one-query-per-call form of the same engine (the "plain" GPU form)
    nsingle = min(args.single, len(queries))
    single_ms = 0.0
    for i in range(nsingle):
        r = eng.solve(queries[i], Ds[i])
        assert r.cost == costs[i], "one-query form disagrees with the batch"
        single_ms += eng.profile()["run_ms"]

    nq = len(queries)
    tot_dev = sum(dev_ms) / 1e3
    tot_wall = sum(wall_s)
    if dist is not None:
        t = torch.tensor([tot_dev, tot_wall], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_dev, tot_wall = float(t[0]), float(t[1])
    value = world * nq * args.steps / tot_dev
    e2e = world * nq * args.steps / tot_wall
    single_qps = nsingle / (single_ms / 1e3) if single_ms > 0 else None
    # the one-per-call sample is the first nsingle queries: comparable with the
    # batch only when every query has the same shape (same k, same kind)
    uniform = len({(len(q), D >= 0) for q, D in zip(queries, Ds)}) == 1

    peak, peak_kind = peaks()
    grow_reads = sums["relax"] / (grow_ms / 1e3) if grow_ms > 0 else None
    gb = grow_bytes(sums)
    achieved = gb / (grow_ms / 1e3) / 1e9 if grow_ms > 0 else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"grow_{args.workload}_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")

    out = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded BA power-law graphs standing in for the reference's external datasets)",
        "config": {"workload": WORKLOADS[args.workload], "queries_per_step_per_gpu": nq,
                   **({"query_filter": f"k={args.k or 'any'} kind={args.kind} first={args.queries or 'all'}"}
                      if (args.k or args.kind != "all" or args.queries) else {}),
                   "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) before every step; "
                   "per-query DP tables (hundreds of MB per step) exceed L2"},
        "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "single_query_qps": single_qps,
        "single_query_sample": f"first {nsingle} queries, one per call" if nsingle else None,
        "batched_over_single": (value / world) / single_qps if single_qps and uniform else None,
        "latency_ms_in_batch": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                                "p99": float(np.percentile(lat, 99))},
        "state_relaxations_per_s": world * sums["relax"] / tot_dev,
        "roofline": {"kernel": "k_grow", "bound": "hbm", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": traffic,
                     "algorithmic_bytes_per_launch": gb / max(grow_launches, 1),
                     "avg_launch_ms": grow_ms / max(grow_launches, 1),
                     "grow_share_of_device_time": grow_ms / (tot_dev * 1e3) if tot_dev else None,
                     "merge_ms": merge_ms,
                     # the grow's target reads are random 4-byte reads: their
                     # rate against a library random gather on the same GPU
                     "random_reads": {"grow_target_reads_per_s": grow_reads,
                                      "ceiling": ceiling,
                                      "frac": grow_reads / ceiling["reads_per_s"] if grow_reads else None}},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = max(1, min(os.cpu_count() or 1, 16))
        qps, times, kind, nproc, nsample, k = cpu_reference_sample(wl, args.workload, procs, procs)
        out["cpu_baseline"] = {
            "value": qps, "unit": "queries/s", "cores": nproc, "kind": kind,
            "sample": f"first {nsample} k={k} queries of this workload, {nproc} single-threaded "
                      f"PrunedDP++ processes on disjoint query ranges (wall clock incl. graph load); "
                      f"reference-internal time per query median "
                      f"{statistics.median(times) if times else float('nan'):.3f} s"}
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
