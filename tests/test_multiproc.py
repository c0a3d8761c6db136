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


def _shard_worker(rank, ws, port, q):
    """One rank of the sharded Hermite schedule: its slice of every call, forces by the FP64
    oracle (the test's force function), gathered over gloo."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import numpy as np
    import torch
    import bench
    from oracle import oracle as O
    dist = bench.dist_init(ws, rank, backend="gloo")
    pgb = bench.load_pkg()
    W, S = pgb.workloads, pgb.shard
    st = W.hermite_state(512, seed=W.SEED0 + 1)          # the same system on every rank
    sets = W.hermite_schedule(512, 6, seed=W.SEED0 + 101)
    sizes = [len(s) for s in sets]
    sl = S.shard_schedule(sizes, ws, rank)
    rows = []
    for c, (lo, hi) in enumerate(sl):
        act = sets[c][lo:hi]
        if len(act) == 0:
            continue
        r = O.g6_force(st.pos[act], st.vel[act], st.idx[act], st.eps2, st.pos, st.vel, st.mass, st.idx)
        rows.append(np.concatenate([r["acc"], r["jrk"], r["pot"][:, None]], 1))
    local = torch.from_numpy(np.concatenate(rows) if rows else np.zeros((0, 7)))
    _, nrows = S.rank_major_order(sizes, ws)
    assert local.shape[0] == nrows[rank]
    got = S.gather_rows(local, nrows, dist).numpy()
    q.put((rank, got))
    dist.destroy_process_group()


def test_two_rank_sharded_hermite_schedule_gathers_the_single_rank_result():
    """The i-partition of a Hermite schedule over two gloo ranks: the slices cover every active
    particle of every call exactly once, and the gathered rows, put back in schedule order, equal
    the single-process result bit for bit (the FP64 oracle as the force function)."""
    import numpy as np
    import torch.multiprocessing as mp
    from conftest import pgb
    from oracle import oracle as O
    W, S = pgb.workloads, pgb.shard
    sets = W.hermite_schedule(512, 6, seed=W.SEED0 + 101)
    sizes = [len(s) for s in sets]
    order, nrows = S.rank_major_order(sizes, 2)
    assert np.array_equal(np.sort(order), np.arange(sum(sizes)))          # every row exactly once
    assert max(nrows) - min(nrows) <= len(sizes)                          # at most one per call apart
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    [p.start() for p in procs]
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])
    [p.join(timeout=60) for p in procs]
    assert all(p.exitcode == 0 for p in procs)
    st = W.hermite_state(512, seed=W.SEED0 + 1)
    act = np.concatenate(sets)
    r = O.g6_force(st.pos[act], st.vel[act], st.idx[act], st.eps2, st.pos, st.vel, st.mass, st.idx)
    ref = np.concatenate([r["acc"], r["jrk"], r["pot"][:, None]], 1)
    for _, got in res:
        back = np.empty_like(got)
        back[order] = got
        assert np.array_equal(back, ref)


def test_cost_partition_covers_every_item_within_the_greedy_bound():
    import numpy as np
    from conftest import pgb
    S = pgb.shard
    rng = np.random.default_rng(3)
    for ws in (2, 3, 8):
        costs = rng.integers(1, 1000, size=257) ** 2
        parts = S.cost_partition(costs, ws)
        allk = np.sort(np.concatenate(parts))
        assert np.array_equal(allk, np.arange(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) <= costs.sum() / ws + costs.max()


def test_contiguous_partition_covers_every_item_within_the_bound():
    import numpy as np
    from conftest import pgb
    S = pgb.shard
    rng = np.random.default_rng(5)
    for ws in (1, 2, 3, 8):
        costs = np.rint(np.exp(rng.uniform(np.log(256), np.log(16384), 1024))) ** 2
        b = S.contiguous_partition(costs, ws)
        assert b[0] == 0 and b[-1] == len(costs) and np.all(np.diff(b) >= 0)
        loads = [costs[b[r]:b[r + 1]].sum() for r in range(ws)]
        assert max(loads) <= costs.sum() / ws + costs.max()
