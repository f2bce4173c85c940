"""Scenario sharding across GPUs (one process per GPU).

Scenarios are independent, so a batch is split across ranks with no communication inside the
Newton loop (weak scaling); results are gathered once at the end.  `shard` balances an
estimated per-scenario cost (e.g. nnz(L+U) x expected iterations for heterogeneous grids) with
longest-processing-time-first assignment; `gather` collects per-rank results on every rank
with one `all_gather_object` (NCCL over NVLink on GPUs, gloo in the CPU tests).
"""

from __future__ import annotations

import heapq

import numpy as np


def shard(n_scen: int, world: int, rank: int, costs=None) -> np.ndarray:
    """Indices of the scenarios rank `rank` of `world` solves (sorted).  Without costs the
    split is contiguous and even; with costs, LPT-greedy on the heaviest scenarios first."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world / rank")
    if costs is None:
        bounds = np.linspace(0, n_scen, world + 1).round().astype(int)
        return np.arange(bounds[rank], bounds[rank + 1])
    costs = np.asarray(costs, dtype=np.float64)
    if costs.shape != (n_scen,):
        raise ValueError("costs must have one entry per scenario")
    heap = [(0.0, r) for r in range(world)]
    owner = np.empty(n_scen, np.int64)
    for s in np.argsort(-costs, kind="stable"):
        load, r = heapq.heappop(heap)
        owner[s] = r
        heapq.heappush(heap, (load + costs[s], r))
    return np.sort(np.nonzero(owner == rank)[0])


def gather(indices, results: dict, n_scen: int, group=None) -> dict:
    """All-gather per-rank results (dict of arrays whose first axis follows `indices`) into
    full arrays of n_scen rows on every rank.  Every rank must call it (collective)."""
    import torch.distributed as dist

    payload = (np.asarray(indices), {k: np.asarray(v) for k, v in results.items()})
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, payload, group=group)
    out = {}
    for idx, res in parts:
        for k, v in res.items():
            if k not in out:
                out[k] = np.zeros((n_scen,) + v.shape[1:], dtype=v.dtype)
            out[k][idx] = v
    return out
