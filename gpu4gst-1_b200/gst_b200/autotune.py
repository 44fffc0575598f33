"""Autotuner of the engine's launch and scheduling parameters (gst_tuning).

The engine's defaults were picked by hand on two workloads.  This module
times candidate values on a given graph and query mix and keeps the fastest,
then writes them to a parameter file that gst_b200.Engine.load_tuning (and
bench.py) apply:

* engine-wide (timed on the whole batch): lanes per grow chunk {8, 16, 32},
  merge and grow of a round in sequence or on two streams, device rounds
  between host polls {4, 8, 16, 32}, queries resident at once;
* per query class (timed on that class's queries alone): (edge, set) pairs
  per grow chunk by (k, plain / D-bounded) {256 .. 4096}, and for plain
  queries the cost-bucket width as a multiple of the typical lightest edge
  {1, 2, 4, 8}.

Search is coordinate descent from the current values, one parameter at a
time, twice over.  Each candidate is timed `repeats` times with the engine's
device timer (CUDA events around the call, gst_engine_profile run_ms) and
scored by the median; a candidate replaces the current value only when it is
faster by more than `margin` (default 1%), so noise does not move the
parameters.  The SM clock is sampled by nvidia-smi during every timing and
its median stored beside the time, so a sample taken at a lower clock shows.
Every candidate's answers must equal the first run's: a parameter may change
speed, never a cost.

    python -m gst_b200.autotune --workload c4 --out gpu4gst-1_b200/tuning/c4.json
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import time

from .clocks import ClockSampler

GROW_LANES = (8, 16, 32)
OVERLAP = (1, 2)
ROUNDS_PER_POLL = (4, 8, 16, 32)
CHUNK_PAIRS = (256, 512, 1024, 2048, 4096)
BUCKET_MULT = (1, 2, 4, 8)


def _class_of(q, D):
    return (len(q), 0 if D < 0 else 1)


class Tuner:
    def __init__(self, engine, queries, Ds, repeats=3, margin=0.01, device=0, log=print):
        self.e = engine
        self.queries = [list(map(int, q)) for q in queries]
        self.Ds = list(map(int, Ds))
        self.repeats = repeats
        self.margin = margin
        self.device = device
        self.log = log
        self.trace = []
        self.ref_costs = {}

    def _time(self, idx, tuning, label):
        """Median device ms of solving the queries `idx` with `tuning` set."""
        self.e.set_tuning(tuning)
        qs = [self.queries[i] for i in idx]
        Ds = [self.Ds[i] for i in idx]
        ms = []
        sampler = ClockSampler(self.device)
        sampler.start()
        for _ in range(self.repeats):
            res = self.e.solve_batch(qs, Ds)
            ms.append(self.e.profile()["run_ms"])
            costs = [r.cost for r in res]
            key = tuple(idx)
            if key not in self.ref_costs:
                self.ref_costs[key] = costs
            elif costs != self.ref_costs[key]:
                raise RuntimeError(f"{label}: costs changed under tuning {tuning}")
        clk = sampler.stop()
        med = statistics.median(ms)
        self.trace.append({"what": label, "tuning": tuning, "ms": ms, "median_ms": med,
                           "sm_mhz": clk.get("sm_mhz"), "reasons": clk.get("reasons")})
        self.log(f"  {label}: {med:.1f} ms (sm {clk.get('sm_mhz')} MHz)")
        return med

    def _descend(self, idx, name, values, current, make, label):
        """Coordinate step: the value of one parameter with the best median
        time; the current value stays unless another beats it by > margin."""
        best_v = current
        best_t = self._time(idx, make(current), f"{label} {name}={current}")
        for v in values:
            if v == current:
                continue
            t = self._time(idx, make(v), f"{label} {name}={v}")
            if t < best_t * (1.0 - self.margin):
                best_v, best_t = v, t
        return best_v, best_t

    def run(self, passes=2):
        t0 = time.time()
        tun = self.e.get_tuning()
        all_idx = list(range(len(self.queries)))
        # warm the engine (slab cache, module load) before any timing
        self.e.solve_batch(self.queries, self.Ds)
        classes = {}
        for i, (q, D) in enumerate(zip(self.queries, self.Ds)):
            classes.setdefault(_class_of(q, D), []).append(i)
        slots_values = sorted({min(1024, v) for v in (64, 128, 256, 512, 1024)})
        for p in range(passes):
            self.log(f"pass {p + 1}: engine-wide parameters on {len(all_idx)} queries")
            tun["grow_lanes"], _ = self._descend(all_idx, "grow_lanes", GROW_LANES, tun["grow_lanes"],
                                                 lambda v: {**tun, "grow_lanes": v}, "all")
            tun["overlap"], _ = self._descend(all_idx, "overlap", OVERLAP, tun["overlap"],
                                              lambda v: {**tun, "overlap": v}, "all")
            tun["rounds_per_poll"], _ = self._descend(all_idx, "rounds_per_poll", ROUNDS_PER_POLL,
                                                      tun["rounds_per_poll"],
                                                      lambda v: {**tun, "rounds_per_poll": v}, "all")
            tun["max_slots"], _ = self._descend(all_idx, "max_slots", slots_values, tun["max_slots"],
                                                lambda v: {**tun, "max_slots": v}, "all")
            self.log(f"pass {p + 1}: per-class parameters")
            for (k, hop), idx in sorted(classes.items()):
                cur = tun["chunk_pairs"][k][hop]

                def with_chunk(v, k=k, hop=hop):
                    cp = [list(x) for x in tun["chunk_pairs"]]
                    cp[k][hop] = v
                    return {**tun, "chunk_pairs": cp}

                best, _ = self._descend(idx, "chunk_pairs", CHUNK_PAIRS, cur, with_chunk,
                                        f"k={k} {'D' if hop else 'plain'}")
                tun["chunk_pairs"][k][hop] = best
                if not hop:
                    def with_mult(v, k=k):
                        bm = list(tun["bucket_mult"])
                        bm[k] = v
                        return {**tun, "bucket_mult": bm}

                    tun["bucket_mult"][k], _ = self._descend(idx, "bucket_mult", BUCKET_MULT,
                                                             tun["bucket_mult"][k], with_mult, f"k={k} plain")
        self.e.set_tuning(tun)
        final = self._time(all_idx, tun, "all (tuned)")
        return {"tuning": tun, "final_median_ms": final, "queries": len(all_idx),
                "classes": {f"k{k}_{'D' if h else 'plain'}": len(v) for (k, h), v in sorted(classes.items())},
                "repeats": self.repeats, "margin": self.margin, "tuner_s": time.time() - t0,
                "trace": self.trace}


def save(path: str, result: dict, workload: str) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    out = {"workload": workload, **result,
           "how": "coordinate descent, median of repeats of the engine's device time per candidate; "
                  "a value changes only when faster by more than the margin"}
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


def load(path: str) -> dict:
    """The tuning dict of a parameter file written by save()."""
    with open(path) as f:
        return json.load(f)["tuning"]


def main():
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    import gst_b200
    from gst_b200 import datagen as dg
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c4", choices=["c2", "c4"])
    ap.add_argument("--out", required=True)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--passes", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    wl = dg.config_c4(1, n_queries=300) if args.workload == "c4" else dg.config_c2(1, n_queries=300)
    e = gst_b200.Engine(device=args.device, profile=True)
    e.load_graph(wl.graph.rowptr, wl.graph.col, wl.graph.w)
    e.load_groups(wl.groups.ptr, wl.groups.mem)
    t = Tuner(e, [q for q, _ in wl.queries], [D for _, D in wl.queries], repeats=args.repeats,
              device=args.device)
    res = t.run(passes=args.passes)
    save(args.out, res, args.workload)
    print(json.dumps({"tuning": res["tuning"], "final_median_ms": res["final_median_ms"],
                      "tuner_s": res["tuner_s"]}))
    e.close()


if __name__ == "__main__":
    main()
