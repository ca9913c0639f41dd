"""Multi-GPU execution: replicas of one world, or shards of independent regions; one process
per GPU.

A single FluidSim world does not shard: a tick is one sorted sweep over one FIFO with one
50k-cell cap, and its pressure searches and flood fills reach anywhere in the world
(fluid.rs:564-657). N GPUs therefore run N replicas of it. Independent regions (a batch of
FluidSims) shard by region with no exchange: each rank steps only its own regions. The only
collective is the timing reduction: the slowest rank's device time and the sum of cell-steps.
"""
from __future__ import annotations


def shard(weights, rank: int, world: int) -> list[int]:
    """Regions of `rank` out of `world`: longest-first greedy balance of the regions' weights
    (resident cells, say). Deterministic; every region goes to exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += float(weights[i])
    return [i for i in range(len(weights)) if owner[i] == rank]


def reduce_rate(dev_ms: float, cells: float, device=None):
    """(max device ms over ranks, total cell-steps over ranks); plain values when not distributed.
    `device` is where the reduction tensor lives (a CUDA device under NCCL, None for CPU/gloo)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(dev_ms), float(cells)
    t = torch.tensor([dev_ms], dtype=torch.float64, device=device)
    c = torch.tensor([cells], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0]), float(c[0])
