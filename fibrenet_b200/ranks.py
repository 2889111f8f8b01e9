"""Work split and timing across ranks (one process per GPU).

A single network does not shard: every rank runs a replica and the job's
rate is all ranks' bead-steps over the slowest rank's time.  Independent
networks (ensembles) are split between ranks by bead count, largest first
onto the least-loaded rank, with no exchange on the data path.
"""
from __future__ import annotations

import heapq


def partition_networks(bead_counts, world: int):
    """Greedy largest-first split of networks over `world` ranks.  Returns a
    list of index lists (network order kept inside each rank)."""
    if world <= 0:
        raise ValueError("world must be positive")
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(bead_counts)), key=lambda i: (-bead_counts[i], i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + bead_counts[i], r))
    return [sorted(p) for p in parts]


def slowest(value: float, dist=None, device=None) -> float:
    """Maximum of `value` over the ranks of the default process group (the
    value itself without one)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def total(value: float, dist=None, device=None) -> float:
    """Sum of `value` over the ranks."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_this_rank: float, elapsed_ms_this_rank: float, dist=None, device=None) -> float:
    """Units per second of the whole job: every rank's units over the
    slowest rank's elapsed time."""
    units = total(units_this_rank, dist, device)
    ms = slowest(elapsed_ms_this_rank, dist, device)
    return units / (ms / 1e3)


def gather_networks(local_indices, local_rows, n_networks: int, dist=None):
    """All-gather of per-network results of a partitioned ensemble: rank r
    holds the rows (one array per network, any shape) of the networks
    ``local_indices``; every rank receives the list of all n_networks rows in
    network order.  Without a process group the local rows are the whole."""
    import numpy as np
    rows = [np.asarray(x) for x in local_rows]
    if len(rows) != len(local_indices):
        raise ValueError("one row per local network")
    pieces = [(list(local_indices), rows)]
    if dist is not None and dist.is_initialized():
        pieces = [None] * dist.get_world_size()
        dist.all_gather_object(pieces, (list(local_indices), rows))
    out = [None] * n_networks
    for idx, rs in pieces:
        for i, r in zip(idx, rs):
            if out[i] is not None:
                raise ValueError(f"network {i} reported by two ranks")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise ValueError(f"networks {missing[:5]} reported by no rank")
    return out
