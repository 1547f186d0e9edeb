"""Replica placement and the once-per-run combination of rank results, on CPU
with world_size-2 gloo process groups (no GPU involved)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dvide_b200 import replicas


def test_partition_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(100), np.log(20000), size=512)).astype(int)
    costs = [replicas.scene_cost(n) for n in sizes]
    for nparts in (1, 2, 4, 8):
        parts = replicas.partition_by_cost(costs, nparts)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT: the heaviest rank exceeds the mean by at most the largest scene
        assert max(loads) - np.mean(loads) <= max(costs) + 1e-9
    assert replicas.partition_by_cost(costs, 4) == replicas.partition_by_cost(costs, 4)


def test_partition_rejects_zero_ranks():
    with pytest.raises(ValueError):
        replicas.partition_by_cost([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        costs = [replicas.scene_cost(n) for n in (500, 20000, 3000, 700, 12000, 100)]
        parts = replicas.partition_by_cost(costs, world)
        mine = parts[rank]
        contacts = 1000.0 * (rank + 1) + len(mine)
        seconds = 0.5 + rank
        s, m = replicas.combine_timed_region(dist, contacts, seconds)
        out[rank] = (tuple(mine), s, m)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    assert set(out.keys()) == {0, 1}
    mine0, s0, m0 = out[0]
    mine1, s1, m1 = out[1]
    assert sorted(mine0 + mine1) == list(range(6)) and not set(mine0) & set(mine1)
    expect = 1000.0 + len(mine0) + 2000.0 + len(mine1)
    assert s0 == s1 == expect
    assert m0 == m1 == 1.5
