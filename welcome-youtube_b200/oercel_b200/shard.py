"""Replica sharding across ranks (one process per GPU).

Replicas are independent boxes, so an ensemble splits across GPUs with no
exchange inside the step: each rank owns a subset of the replicas, balanced
by bead count (longest-processing-time greedy: largest replica first, onto the
least-loaded rank).  The one exchange of the batched adjoint, the shared
parameter gradient, is a sum over ranks (reduce_gradients).
"""
from __future__ import annotations


def shard_replicas(n_beads, world_size):
    """list of replica indices per rank; deterministic, every replica exactly once"""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(n_beads)), key=lambda r: (-int(n_beads[r]), r))
    load = [0] * world_size
    parts = [[] for _ in range(world_size)]
    for r in order:
        k = min(range(world_size), key=lambda q: (load[q], q))
        parts[k].append(r)
        load[k] += int(n_beads[r])
    return [sorted(p) for p in parts]


def my_replicas(n_beads, rank, world_size):
    return shard_replicas(n_beads, world_size)[rank]


def reduce_gradients(grad, group=None):
    """sum a tensor over all ranks in place: the one exchange of a batched fit
    (the shared parameter gradient and the loss).  gloo reduces CPU tensors as
    they are; under NCCL a CPU tensor travels through a CUDA copy."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return grad
    if dist.get_backend(group) == "nccl" and not grad.is_cuda:
        import torch
        t = grad.to(torch.device("cuda", torch.cuda.current_device()))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        grad.copy_(t.cpu())
    else:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def replica_share(reps, rank, world_size):
    """this rank's part of an ensemble given as (Params, n_beads) pairs: the
    replicas shard_replicas assigns to it, in ensemble order, with their
    indices in the whole ensemble"""
    idx = my_replicas([n for _, n in reps], rank, world_size)
    return idx, [reps[i] for i in idx]
