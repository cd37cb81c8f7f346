"""Shot-sharded FWI over several GPUs: one process and one engine context per GPU.

The path shards by shot: forward, replay, adjoint and per-shot preconditioning of one shot
touch no other shot.  Each rank holds the whole model and a share of the shots; the one
exchange per gradient is the FP64 stack of the gradient and pseudo-Hessian (the
reference's shot loop, propagation.c:953-976) plus the scalar sums of the FWI loop (misfit
and step length, optimization.c:13-132).  The engine calls an all-reduce hook at exactly
those points (``Context.set_allreduce``); after the stack every rank runs the global
preconditioning, smoothing, perturbation and model update redundantly on identical data, so
all ranks keep identical models.

``shard`` assigns shots to ranks, ``device_hook`` is the hook for NCCL process groups
(torch.distributed), ``allreduce_`` the in-place sum it uses (also usable on CPU tensors
with gloo).
"""
from __future__ import annotations

from typing import Callable, Sequence


def shot_cost(shot) -> int:
    """Relative cost of one shot: its window width times its record length (the padded
    window's rows are the same for every shot of a model, and nt is the record length)."""
    return (int(shot.ix_max) - int(shot.ix_min) + 1) * int(shot.ns)


def shard(shots: Sequence, world: int, rank: int, cost: Callable | None = None) -> list[int]:
    """Indices of the shots that ``rank`` of ``world`` runs, in survey order.

    Longest-processing-time assignment: shots in decreasing cost (ties in survey order) go to
    the rank with the least work so far (ties to the lowest rank), which keeps equal-cost
    surveys round-robin and bounds the imbalance by one shot.  Deterministic: every rank
    computes the same partition.  Each rank gets at least one shot when len(shots) >= world."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    cost = cost or shot_cost
    order = sorted(range(len(shots)), key=lambda i: (-cost(shots[i]), i))
    load = [0] * world
    owner = [0] * len(shots)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += cost(shots[i])
    return [i for i in range(len(shots)) if owner[i] == rank]


def allreduce_(t):
    """In-place sum of a tensor over the default process group (NCCL for CUDA tensors over
    NVLink, gloo for CPU tensors)."""
    import torch.distributed as dist

    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t


class _DeviceDoubles:
    """A zero-copy view of ``count`` device doubles for torch.as_tensor."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_hook(device: int):
    """Exchange hook for ``Context.set_allreduce`` on a NCCL process group: views the engine's
    FP64 buffer as a CUDA tensor and sums it over the ranks on the engine's stream (the
    collective starts after the engine's prior work on that stream, and the engine's later
    work waits for it)."""
    import torch

    def hook(ptr: int, count: int, stream: int):
        t = torch.as_tensor(_DeviceDoubles(ptr, count), device=f"cuda:{device}")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=f"cuda:{device}")):
            allreduce_(t)

    return hook
