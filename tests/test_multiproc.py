"""Multi-process plumbing of the benchmark on CPU (world size 2, gloo, 127.0.0.1).

Every rank runs its own replica of the workload (independent work items, no data-path
collective); the only collectives are the max / sum of scalar timings and pair counts over
ranks, which this test exercises with the same helpers bench.py uses under torchrun.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import bench
    dist = bench.dist_init(ws, rank, backend="gloo")
    pgb = bench.load_pkg()
    W = pgb.workloads
    sets = W.hermite_schedule(4096, 8, seed=W.SEED0 + 101 + rank)   # each rank its own replica
    t = 1.0 + rank                                                   # rank 1 is the slowest
    tmax = bench.reduce_max(t, ws, torch.device("cpu"))
    total = bench.reduce_sum(float(sum(len(s) for s in sets)), ws, torch.device("cpu"))
    bench.barrier(ws)
    q.put((rank, tmax, total, [len(s) for s in sets]))
    dist.destroy_process_group()


def test_two_rank_gloo_reduction():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    [p.start() for p in procs]
    res = sorted(q.get(timeout=120) for _ in procs)
    [p.join(timeout=60) for p in procs]
    assert all(p.exitcode == 0 for p in procs)
    (_, tmax0, tot0, s0), (_, tmax1, tot1, s1) = res
    assert tmax0 == tmax1 == 2.0                    # max over ranks
    assert tot0 == tot1 == float(sum(s0) + sum(s1))   # sum over ranks
    assert s0 != s1                                 # independent replicas
