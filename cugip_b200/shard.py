"""Multi-GPU batches: instances are independent graphs, so they shard across
ranks (one process per GPU) with no exchange while solving; only the int64
flows (and, on request, the cut masks) are gathered at the end.

The reference has no multi-GPU path; this follows the one-process-per-GPU
model with torch.distributed for the plumbing (NCCL on GPUs, gloo in the CPU
tests).
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def partition_lpt(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Longest-processing-time-first partition of instance indices over
    `world` ranks by voxel count (deterministic: ties go to the lower rank)."""
    if world <= 0:
        raise ValueError("world must be positive")
    heap = [(0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    for p in parts:
        p.sort()
    return parts


def solve_sharded(extents: Sequence[Sequence[int]], solve_local: Callable[[list[int]], list[int]],
                  group=None) -> list[int]:
    """Solves the instances assigned to this rank with `solve_local(indices)`
    (which returns their flows in the same order) and gathers every flow on
    every rank.  Collectives are the same on all ranks in the same order."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    sizes = [int(x) * int(y) * int(z) for x, y, z in extents]
    parts = partition_lpt(sizes, world)
    mine = parts[rank]
    flows_local = solve_local(mine) if mine else []
    if len(flows_local) != len(mine):
        raise RuntimeError("solve_local returned a wrong number of flows")
    if world == 1:
        return list(flows_local)
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (mine, list(flows_local)), group=group)
    flows = [0] * len(extents)
    for idx, fl in gathered:
        for i, f in zip(idx, fl):
            flows[i] = int(f)
    return flows


def solve_batch_on_rank(volumes, policy=None) -> list[int]:
    """solve_local for cugip_b200 volumes: one batched solve of the given volumes
    on this rank's GPU."""
    from .graph_cut import Batch
    B = Batch([(v.X, v.Y, v.Z) for v in volumes])
    try:
        for i, v in enumerate(volumes):
            B.set_tweights(i, v.capS, v.capT)
            for ax in range(3):
                B.set_nweights(i, ax, v.n[ax])
        return B.max_flow(policy)
    finally:
        B.close()
