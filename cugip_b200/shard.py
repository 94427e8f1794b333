"""Multi-GPU batches: instances are independent graphs, so they shard across
ranks (one process per GPU) by voxel count (LPT) with no exchange while
solving; the int64 flows are gathered on every rank at the end, and on
request the cut masks on one rank.

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


def solve_sharded(extents: Sequence[Sequence[int]], solve_local: Callable, group=None,
                  masks_to: int | None = None):
    """Solves the instances assigned to this rank with `solve_local(indices)`
    and gathers every flow on every rank; returns the list of all flows.

    `solve_local` returns the flows of its instances in the given order, or,
    with `masks_to` set, a pair (flows, masks) where masks[k] is the pair of
    cut sets (source side, sink side; uint8 arrays) of instance indices[k].
    Then the masks of every instance are also gathered on rank `masks_to`, and
    the call returns (flows, masks) there ((flows, None) on the other ranks).
    Every rank takes the same collective steps in the same order."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    sizes = [int(x) * int(y) * int(z) for x, y, z in extents]
    parts = partition_lpt(sizes, world)
    mine = parts[rank]
    res = solve_local(mine) if mine else (([], []) if masks_to is not None else [])
    flows_local, masks_local = (res if masks_to is not None else (res, None))
    if len(flows_local) != len(mine) or (masks_local is not None and len(masks_local) != len(mine)):
        raise RuntimeError("solve_local returned a wrong number of results")
    flows = [0] * len(extents)
    if world == 1:
        for i, f in zip(mine, flows_local):
            flows[i] = int(f)
        gathered_masks = [(mine, list(masks_local))] if masks_local is not None else None
    else:
        gathered: list = [None] * world
        dist.all_gather_object(gathered, (mine, [int(f) for f in flows_local]), group=group)
        for idx, fl in gathered:
            for i, f in zip(idx, fl):
                flows[i] = f
        gathered_masks = None
        if masks_to is not None:
            objs = [None] * world if rank == masks_to else None
            dist.gather_object((mine, list(masks_local)), objs, dst=masks_to, group=group)
            gathered_masks = objs
    if masks_to is None:
        return flows
    if rank != masks_to:
        return flows, None
    masks: list = [None] * len(extents)
    for idx, ms in gathered_masks:
        for i, m in zip(idx, ms):
            masks[i] = m
    return flows, masks


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
