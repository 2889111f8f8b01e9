"""A partitioned ensemble across ranks equals one batched run, bit for bit.

Two processes (gloo for the host-side gather), both on cuda:0: each uploads
its partition_networks share of a small ensemble of tensile networks into
one context, records every network's reaction curve (the clamp force after
each fn_step(every) call) and the per-network results are all-gathered.
Their kernels never wait on each other; only the gather crosses ranks.  The
gathered curves must equal those of all networks batched in one process.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

SAMPLES, EVERY = 12, 10


def ensemble():
    from fibrenet_b200 import generate as g
    out = []
    for k, F in enumerate([12, 40, 25, 60, 18]):
        side = 1000.0 * np.sqrt(F / 20000.0)
        out.append(g.tensile_network(seed=40 + k, fibres=F, beads=20, box=(side, side, 10.0),
                                     z_range=(1.0, 9.0), clamp_lo=2.0, clamp_hi=side - 2.0, pull=0.5,
                                     fail_mu=np.log(0.5), fail_sigma=0.4))
    return out


def curves(models, device=0):
    from fibrenet_b200.native import Simulation
    rows = [np.zeros((SAMPLES, 3)) for _ in models]
    with Simulation(models, device=device, list_capacity=64, reorder=True) as s:
        for t in range(SAMPLES):
            s.step(EVERY)
            for k in range(len(models)):
                rows[k][t] = s.observe(k, reaction_type=2)["reaction"]
    return rows


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from fibrenet_b200.ranks import gather_networks, partition_networks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        ms = ensemble()
        mine = partition_networks([m.n_beads for m in ms], world)[rank]
        rows = curves([ms[i] for i in mine])
        out[rank] = (mine, gather_networks(mine, rows, len(ms), dist))
    finally:
        dist.destroy_process_group()


def test_partitioned_ensemble_equals_one_batched_run():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    want = curves(ensemble())
    assert any(np.abs(w).sum() > 0 for w in want)
    parts = [out[0][0], out[1][0]]
    assert parts[0] and parts[1] and sorted(parts[0] + parts[1]) == list(range(len(want)))
    for r in range(2):
        got = out[r][1]
        assert len(got) == len(want)
        for k in range(len(want)):
            np.testing.assert_array_equal(got[k], want[k], err_msg=f"rank {r} network {k}")
