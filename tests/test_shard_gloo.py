"""Replica sharding and the shared-gradient reduction with world_size 2 (gloo on CPU)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oercel_b200.shard import reduce_gradients, shard_replicas
from oercel_b200 import workloads


def test_shard_covers_every_replica_once_and_balances():
    nb = [n for _, n in workloads.config3(n_replicas=256, chem=False)]
    for ws in (1, 2, 3, 8):
        parts = shard_replicas(nb, ws)
        flat = sorted(r for p in parts for r in p)
        assert flat == list(range(len(nb)))
        loads = [sum(nb[r] for r in p) for p in parts]
        assert max(loads) - min(loads) <= max(nb)
    assert shard_replicas([5, 5, 5], 2) == shard_replicas([5, 5, 5], 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, nb, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_replicas(nb, world)[rank]
        # each rank's "gradient": one row per replica it owns, summed
        g = torch.zeros(18, dtype=torch.float64)
        for r in mine:
            g += torch.arange(18, dtype=torch.float64) * (r + 1)
        reduce_gradients(g)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out[rank] = (g.tolist(), gathered)
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    nb = [n for _, n in workloads.config3(n_replicas=16, chem=False)]
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), nb, out), nprocs=world, join=True)
    want = (torch.arange(18, dtype=torch.float64) * sum(r + 1 for r in range(len(nb)))).tolist()
    for rank in range(world):
        g, gathered = out[rank]
        assert g == pytest.approx(want)
        assert sorted(r for p in gathered for r in p) == list(range(len(nb)))
