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


class StubEngine:
    """The engine interface the window Function and fit use, on the CPU: replica
    r's loss is (r + 1) / 2 ((a_W_T - 70)^2 + (gamma - 4)^2), its gradient row
    holds (r + 1) (a_W_T - 70) and (r + 1) (gamma - 4) in their slots."""

    def __init__(self, replicas):
        from oercel_b200 import Params
        self.replicas = list(replicas)
        self.nrep = len(self.replicas)
        self.params = [Params(a_W_T=60, gamma=4.5) for _ in self.replicas]
        self.n_beads = [8] * self.nrep
        self.step_no = 0

    def set_params(self, r, p):
        self.params[r] = p

    def forces(self, step):
        pass

    def window_adjoint(self, nsteps, ckpt, spec, target):
        import numpy as np
        from oercel_b200 import fit
        loss = np.zeros(self.nrep)
        grad = np.zeros((self.nrep, fit.NGRAD))
        for k, r in enumerate(self.replicas):
            a, g = self.params[k].a[0][2], self.params[k].gamma
            loss[k] = (r + 1) / 2 * ((a - 70.0) ** 2 + (g - 4.0) ** 2)
            grad[k, fit.param_index("a_W_T")] = (r + 1) * (a - 70.0)
            grad[k, fit.param_index("gamma")] = (r + 1) * (g - 4.0)
        self.step_no += nsteps
        return loss, grad, np.zeros((self.nrep, spec.nbin))


def _fit_run(replicas, distributed):
    from oercel_b200 import Engine, fit
    eng = StubEngine(replicas)
    spec = Engine.rdf_spec(nbin=4)
    hist = fit.fit(eng, ["a_W_T", "gamma"], [0.0] * 4, iters=4, window=10, ckpt=5, spec=spec, lr=0.5,
                   distributed=distributed)
    return [(h["loss"], h["grad"], h["values"]) for h in hist]


def _fit_worker(rank, world, port, nb, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = _fit_run(shard_replicas(nb, world)[rank], True)
    finally:
        dist.destroy_process_group()


def test_two_ranks_fit_takes_the_single_rank_step():
    """fit with distributed=True on 2 gloo ranks, each holding its share of 5
    replicas: both ranks take the identical Adam steps, equal to one rank
    holding all 5 (the summed gradient)"""
    nb = [100, 300, 200, 500, 400]
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_fit_worker, args=(world, _free_port(), nb, out), nprocs=world, join=True)
    want = _fit_run(range(len(nb)), False)
    assert out[0] == out[1]
    for (l, g, v), (lw, gw, vw) in zip(out[0], want):
        assert l == pytest.approx(lw, rel=1e-12)
        assert g == pytest.approx(gw, rel=1e-12)
        assert v == pytest.approx(vw, rel=1e-12)
    assert want[-1][2][0] > 60.0 and want[-1][2][1] < 4.5  # Adam moves both toward the minimum
