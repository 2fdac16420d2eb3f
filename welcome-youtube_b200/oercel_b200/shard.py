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
    """sum a gradient tensor over all ranks in place (NCCL for CUDA tensors, gloo for CPU)"""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad
