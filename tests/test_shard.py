"""Multi-GPU batch sharding: host logic, and the gather across two ranks over
gloo on the CPU (the solve itself is faked; every rank runs the same
collectives in the same order)."""
import os

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


def _fake_flow(i):
    return 1000 + 7 * i


def _worker(rank, world, port, extents, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seen = []

        def solve_local(idx):
            seen.extend(idx)
            return [_fake_flow(i) for i in idx]

        flows = solve_sharded(extents, solve_local)
        out[rank] = (flows, seen)
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
        flows, seen = res[r]
        assert flows == expected
        seen_all += seen
    assert sorted(seen_all) == list(range(len(extents)))  # every instance solved exactly once
