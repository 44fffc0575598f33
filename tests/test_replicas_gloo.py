"""Multi-rank query sharding on CPU (gloo, world size 2).

The multi-GPU form is replicas: disjoint query shares per rank and a gather of
the small results.  This checks the host logic with two gloo ranks and a CPU
stand-in solver (the oracle), so no GPU is needed."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gst_b200 import replicas


def test_shard_is_a_balanced_partition():
    qs = [[0, 1, 2]] * 5 + [[0, 1, 2, 3, 4, 5, 6]] * 3 + [[1, 2, 3, 4, 5]] * 4
    Ds = [-1, 2, -1, 3, -1, -1, 4, -1, 2, -1, -1, 5]
    for world in (1, 2, 3, 4):
        parts = replicas.shard(qs, Ds, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(qs)))
        loads = [sum(replicas.query_weight(len(qs[i]), Ds[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(replicas.query_weight(len(q), d) for q, d in zip(qs, Ds))
    assert replicas.shard(qs, Ds, 2) == replicas.shard(qs, Ds, 2)  # same on every rank


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_q):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(here, "gpu4gst-1_b200"))
    sys.path.insert(0, here)
    from gst_b200 import datagen as dg
    from gst_b200 import replicas as rp
    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = dg.ba_graph(300, 3, 1, 30, seed=7)
    gr = dg.make_groups(g.V, 30, seed=8, uniform=(1, 5))
    qs = [list(q) for q, _ in dg.make_queries(gr.n, 10, [2, 3, 4], seed=9)]
    Ds = [-1, 2, -1, 3, -1, 2, -1, -1, 4, -1]
    calls = []

    class R:
        def __init__(self, c):
            self.cost, self.feasible = c, c < oracle.INF

    def cpu_solve(batch, bDs):
        calls.append(len(batch))
        return [R(oracle.dpbf(g, gr, q)[0] if d < 0 else oracle.hop(g, gr, q, d)[0]) for q, d in zip(batch, bDs)]

    got = rp.solve_sharded(cpu_solve, qs, Ds)
    want = [cpu_solve([q], [d])[0].cost for q, d in zip(qs, Ds)]
    out_q.put((rank, [c for c, _ in got] == want, calls[0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_query_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert all(ok for _, ok, _ in res)
    assert sum(n for _, _, n in res) == 10  # each query solved by exactly one rank
