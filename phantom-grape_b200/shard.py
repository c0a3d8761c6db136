"""Multi-GPU partitioning of the force workloads: one process per GPU, no data-path collective
except the gather of the results.

The reference parallelises the same way inside one host: its OpenMP builds split the
i-particles of a call over threads that share one j-memory (PG6/libpg6/phantom_g6.c:194-198;
PG5/newton/libpg5/phantom_g5.c:315-348 over ``*MC(tid)``).  Here the ranks are processes on
separate GPUs:

* Hermite calls (one active set against every j): every rank holds the whole j-memory and
  predicts it itself (the predictor is O(N) per call against O(N x active) for the force), and
  computes a contiguous slice of each call's active set (:func:`split_range`).  The slices of
  all calls are concatenated per rank (rank-major order), so one all-gather returns every
  result; :func:`rank_major_order` maps them back to the schedule's order.
* Independent work items (TreePM groups, tree groups, clusters): items are assigned to ranks by
  their estimated cost, longest first to the least-loaded rank (:func:`cost_partition`), or in
  contiguous ranges of about equal cost (:func:`contiguous_partition`) where a rank's caller
  takes an index range; each rank runs its items in one batched launch and the results are
  gathered the same way.

:func:`gather_rows` is the only collective: an all-gather of rows padded to the largest rank's
count (NCCL on GPU tensors, gloo on CPU tensors).
"""
from __future__ import annotations

import numpy as np


def split_range(n: int, ws: int, rank: int) -> tuple[int, int]:
    """The contiguous share [lo, hi) of rank `rank` out of n items split over ws ranks (sizes
    differ by at most one)."""
    return (n * rank) // ws, (n * (rank + 1)) // ws


def shard_schedule(set_sizes, ws: int, rank: int):
    """Per call c of a Hermite schedule (active sets of set_sizes[c] particles): the slice
    [lo_c, hi_c) of the call's active set that `rank` computes.  Returns an int array [ncalls, 2]."""
    return np.array([split_range(int(n), ws, rank) for n in set_sizes], dtype=np.int64).reshape(-1, 2)


def rank_major_order(set_sizes, ws: int):
    """Positions, in the schedule's concatenated order (call by call, the active set's order),
    of the rows of a rank-major gather: rank 0's slices of calls 0, 1, ..., then rank 1's, ...
    Returns (order, rows) where order[k] is the schedule row of gathered row k (pads removed) and
    rows[r] the number of rows of rank r."""
    off = np.concatenate([[0], np.cumsum(np.asarray(set_sizes, dtype=np.int64))])
    order, rows = [], []
    for r in range(ws):
        sl = shard_schedule(set_sizes, ws, r)
        idx = [np.arange(off[c] + lo, off[c] + hi) for c, (lo, hi) in enumerate(sl)]
        idx = np.concatenate(idx) if idx else np.zeros(0, np.int64)
        order.append(idx)
        rows.append(len(idx))
    return np.concatenate(order), rows


def cost_partition(costs, ws: int):
    """Assign items with estimated costs to ws ranks: longest first, each to the rank with the
    least load so far (ties to the lower rank).  Returns a list of ws sorted index arrays.
    The largest load is at most sum(costs)/ws + max(costs) (the greedy bound)."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(ws)
    parts = [[] for _ in range(ws)]
    for k in order:
        r = int(np.argmin(load))
        parts[r].append(int(k))
        load[r] += costs[k]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def contiguous_partition(costs, ws: int):
    """Split a sequence of items into ws contiguous ranges of about equal cost: range r ends at
    the first item where the running cost reaches (r+1)/ws of the total.  Returns ws + 1
    boundaries; the largest range costs at most sum(costs)/ws + max(costs).  For items whose
    per-rank callers take an index range (the plain API's per-cluster loop)."""
    c = np.cumsum(np.asarray(costs, dtype=np.float64))
    total = c[-1] if len(c) else 0.0
    b = [0]
    for r in range(1, ws):
        b.append(int(np.searchsorted(c, total * r / ws, side="left")) + 1 if len(c) else 0)
        b[-1] = min(max(b[-1], b[-2]), len(c))
    b.append(len(c))
    return np.array(b, dtype=np.int64)


def gather_rows(local, rows, dist, group=None):
    """All-gather of per-rank row blocks: `local` holds this rank's rows[rank] rows (a torch
    tensor, first dimension = rows, any row shape); returns the rank-major concatenation of every
    rank's rows on every rank (pads dropped).  With one rank it returns `local` itself."""
    import torch
    ws = len(rows)
    if ws == 1:
        return local
    rmax = max(rows)
    shape = tuple(local.shape[1:])
    pad = torch.zeros((rmax,) + shape, dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty((rmax,) + shape, dtype=local.dtype, device=local.device) for _ in range(ws)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([bufs[r][:rows[r]] for r in range(ws)])
