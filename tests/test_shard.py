"""Multi-GPU batch sharding: host logic, and the gather across two ranks over
gloo on the CPU (the solve itself is faked; every rank runs the same
collectives in the same order)."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cugip_b200.shard import partition_lpt, solve_sharded


def test_lpt_partition_is_balanced_and_complete():
    sizes = [100, 90, 80, 70, 60, 50, 40, 30, 20, 10]
    parts = partition_lpt(sizes, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert partition_lpt(sizes, 3) == parts  # deterministic
    assert partition_lpt([5], 4) == [[0], [], [], []]
    with pytest.raises(ValueError):
        partition_lpt(sizes, 0)


@pytest.mark.parametrize("world", [2, 3, 4, 8])
def test_lpt_shards_of_the_96_instance_batch_are_balanced(world):
    """The real 96 extents (32..160 per axis): every rank's voxel load is within
    the largest instance of every other rank's."""
    from cugip_b200 import volume
    ext = [(s.X, s.Y, s.Z) for s in (volume.preset(4, i) for i in range(96))]
    sizes = [x * y * z for x, y, z in ext]
    parts = partition_lpt(sizes, world)
    assert sorted(i for p in parts for i in p) == list(range(96))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert max(loads) <= sum(sizes) / world + max(sizes)


def _fake_flow(i):
    return 1000 + 7 * i


def _fake_masks(i, n):
    return (np.full(n, i % 2, np.uint8), np.arange(n, dtype=np.uint8) + i)


def _worker(rank, world, port, extents, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def solve_local(idx):
            seen.extend(idx)
            return [_fake_flow(i) for i in idx]

        flows = solve_sharded(extents, solve_local)

        def solve_local_masks(idx):
            return ([_fake_flow(i) for i in idx],
                    [_fake_masks(i, extents[i][0] * extents[i][1] * extents[i][2]) for i in idx])

        flows2, masks = solve_sharded(extents, solve_local_masks, masks_to=1)
        sums = None if masks is None else [(int(a.sum()), int(b.astype(np.int64).sum())) for a, b in masks]
        out[rank] = (flows, seen, flows2, sums)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_gather_over_gloo(world):
    extents = [(32 + 8 * i, 40, 33 + i) for i in range(11)]
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, extents, out), nprocs=world, join=True)
        res = dict(out)
    expected = [_fake_flow(i) for i in range(len(extents))]
    seen_all = []
    for r in range(world):
        flows, seen, flows2, sums = res[r]
        assert flows == expected and flows2 == expected
        seen_all += seen
        if r == 1:  # the masks of every instance arrive on rank 1, in instance order
            want = []
            for i, (x, y, z) in enumerate(extents):
                a, b = _fake_masks(i, x * y * z)
                want.append((int(a.sum()), int(b.astype(np.int64).sum())))
            assert sums == want
        else:
            assert sums is None
    assert sorted(seen_all) == list(range(len(extents)))  # every instance solved exactly once
