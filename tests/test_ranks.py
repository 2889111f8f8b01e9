"""Rank logic of the replica / ensemble split, on the CPU with gloo."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from fibrenet_b200.ranks import gather_networks, job_rate, partition_networks, slowest


def test_partition_balances_and_covers():
    counts = [100_000, 2_500, 50_000, 75_000, 30_000, 30_000, 90_000, 10_000]
    parts = partition_networks(counts, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(counts)))
    loads = [sum(counts[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(counts)
    assert partition_networks(counts, 1) == [list(range(len(counts)))]
    with pytest.raises(ValueError):
        partition_networks(counts, 0)


def test_single_process_passthrough():
    assert slowest(3.5) == 3.5
    assert job_rate(1000, 500.0) == 2000.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r processed (r + 1) * 1000 bead-steps in (r + 1) * 100 ms
        rate = job_rate((rank + 1) * 1000.0, (rank + 1) * 100.0, dist)
        out[rank] = (rate, slowest(rank * 7.0, dist))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    # (1000 + 2000) bead-steps over the slowest 200 ms
    assert out[0] == out[1] == (15000.0, 7.0)


def _worker_leaves(rank, world, port, out):
    import datetime
    import time

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        # leaves between steps, with no collective of its own in flight
        os._exit(0)
    t0 = time.monotonic()
    try:
        job_rate(1000.0, 100.0, dist)
        out[rank] = ("no error", time.monotonic() - t0)
    except Exception as e:  # noqa: BLE001 - any error ends the wait
        out[rank] = (type(e).__name__, time.monotonic() - t0)
    os._exit(0)


def test_rank_that_leaves_ends_the_others_collective_with_an_error():
    """A rank that exits between steps: the remaining rank's next timing
    collective returns an error within the process group's short timeout
    instead of waiting for good."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker_leaves, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    what, waited = out[0]
    assert what != "no error"
    assert waited < 60.0


def _worker_gather(rank, world, port, out):
    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        counts = [500, 4000, 1200, 3000, 800, 2500, 100]
        mine = partition_networks(counts, world)[rank]
        # every network's "curve" is a function of its index alone
        rows = [np.full((3, 2), 10.0 * i + 0.5) for i in mine]
        allrows = gather_networks(mine, rows, len(counts), dist)
        out[rank] = [float(r[0, 0]) for r in allrows]
    finally:
        dist.destroy_process_group()


def test_gather_networks_over_two_gloo_ranks():
    """Per-network results of a partitioned ensemble come back to every rank
    in network order."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker_gather, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    want = [10.0 * i + 0.5 for i in range(7)]
    assert out[0] == out[1] == want


def test_gather_networks_rejects_gaps_and_duplicates():
    import numpy as np
    with pytest.raises(ValueError):
        gather_networks([0, 2], [np.zeros(1), np.zeros(1)], 3)
    assert [float(x[0]) for x in gather_networks([1, 0], [np.ones(1), np.zeros(1)], 2)] == [0.0, 1.0]
