"""Device-resident batches (bound inputs/outputs, enqueue, CUDA graph replay)
and the autotuner, checked against the golden fixtures."""
import json
import os

import numpy as np
import pytest

from cugip_b200 import volume
from cugip_b200.graph_cut import SINK, SOURCE, Batch, GridGraph, Policy, autotune_lookup
from tests.gpu_helpers import sha

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")))
CASES = {(c["workload"], c["index"]): c for c in GOLDEN["cases"]}
KEYS = [(4, i) for i in range(8)] + [(1, 0)]


@pytest.fixture(scope="module")
def device_batch():
    import torch
    vols = [volume.workload(*k) for k in KEYS]
    dev = torch.device("cuda", 0)
    ins = [[torch.from_numpy(a).to(dev) for a in v.arrays()] for v in vols]
    outs = [(torch.zeros(v.N, dtype=torch.uint8, device=dev), torch.zeros(v.N, dtype=torch.uint8, device=dev))
            for v in vols]
    flows = torch.zeros(len(vols), dtype=torch.int64, device=dev)
    B = Batch([(v.X, v.Y, v.Z) for v in vols])
    for i, (d, o) in enumerate(zip(ins, outs)):
        B.bind_inputs(i, d[0].data_ptr(), d[1].data_ptr(), [t.data_ptr() for t in d[2:]])
        B.bind_outputs(i, o[0].data_ptr(), o[1].data_ptr())
    yield B, vols, ins, outs, flows
    B.close()


def _check(outs, flows_host):
    for i, k in enumerate(KEYS):
        c = CASES[k]
        assert flows_host[i] == c["flow"], k
        assert sha(outs[i][0].cpu().numpy()) == c["smin_sha256"], k
        assert sha(outs[i][1].cpu().numpy()) == c["treach_sha256"], k


def test_enqueue_matches_golden(device_batch):
    B, vols, ins, outs, flows = device_batch
    for o in outs:
        o[0].fill_(7); o[1].fill_(7)
    B.enqueue(Policy(), flows.data_ptr())
    fl = B.wait()
    assert fl == [int(x) for x in flows.cpu()]
    _check(outs, fl)


@pytest.mark.parametrize("policy", [Policy(), Policy(local_pulses=2, region_relabels=4, sweeps_per_relabel=4, ctas_per_sm=3),
                                    Policy(ctas_per_sm=3, stall_sweeps=1, sweeps_per_relabel=64),
                                    Policy(ctas_per_sm=4, region_relabels=-1, local_pulses=8),
                                    Policy(ctas_per_sm=4, region_relabels=4),
                                    Policy(ctas_per_sm=4, region_relabels=4, bfs_warp_min=8),
                                    Policy(exclusive=1, ctas_per_sm=4, region_relabels=4, bfs_warp_min=8),
                                    Policy(exclusive=1, local_pulses=2, sweeps_per_relabel=3)])
def test_graph_replay_matches_golden(device_batch, policy):
    B, vols, ins, outs, flows = device_batch
    B.graph_create(policy, flows.data_ptr())
    for rep in range(3):
        for o in outs:
            o[0].fill_(7); o[1].fill_(7)
        flows.fill_(-1)
        B.graph_launch()
        fl = B.wait()
        assert fl == [int(x) for x in flows.cpu()]
        _check(outs, fl)


def test_graph_picks_up_new_capacities(device_batch):
    """The graph reads the bound buffers on every replay: overwrite instance 0
    with all-zero capacities and its flow drops to 0."""
    B, vols, ins, outs, flows = device_batch
    B.graph_create(Policy(), flows.data_ptr())
    saved = [t.clone() for t in ins[0]]
    for t in ins[0]:
        t.zero_()
    B.graph_launch()
    fl = B.wait()
    assert fl[0] == 0 and fl[1:] == [CASES[k]["flow"] for k in KEYS[1:]]
    for t, s in zip(ins[0], saved):
        t.copy_(s)
    B.graph_launch()
    _check(outs, B.wait())


def test_autotune_batch_and_lookup(device_batch):
    B, vols, ins, outs, flows = device_batch
    cands = [Policy(local_pulses=L, region_relabels=R, sweeps_per_relabel=K) for L, R, K in
             ((2, 4, 4), (4, 2, 8), (8, 1, 8))]
    best, ms = B.autotune(cands, repeats=1)
    assert ms > 0 and best.local_pulses in (2, 4, 8)
    got = autotune_lookup(sum(v.N for v in vols), len(vols))
    assert got is not None and got.local_pulses == best.local_pulses
    B.enqueue(best, flows.data_ptr())
    _check(outs, B.wait())


def test_autotune_grid_keeps_capacities():
    v = volume.workload(1)
    g = GridGraph(v.X, v.Y, v.Z)
    g.set_tweights(v.capS, v.capT)
    for ax in range(3):
        g.set_nweights(ax, v.n[ax])
    best, ms = g.autotune(repeats=1)  # built-in candidate grid
    assert ms > 0
    c = CASES[(1, 0)]
    assert g.max_flow(best) == c["flow"]
    assert sha(g.fill_segments(mask=1, which=SOURCE)) == c["smin_sha256"]
    assert sha(g.fill_segments(mask=1, which=SINK)) == c["treach_sha256"]
    g.close()


def test_sharded_solve_single_rank_matches_golden():
    from cugip_b200.shard import solve_batch_on_rank, solve_sharded
    keys = [(4, i) for i in range(5)]
    vols = [volume.workload(*k) for k in keys]
    flows = solve_sharded([(v.X, v.Y, v.Z) for v in vols], lambda idx: solve_batch_on_rank([vols[i] for i in idx]))
    assert flows == [CASES[k]["flow"] for k in keys]


def test_bound_inputs_are_checked_like_host_uploads():
    """The device-resident path refuses negative capacities and capacities
    that could overflow int32 excess or residuals, like the host setters, and
    matches the oracle on asymmetric bound n-links."""
    import torch
    from cugip_b200 import _lib
    from oracle import oracle  # the checker
    from tests import graphs
    dev = torch.device("cuda", 0)
    X, Y, Z = 11, 9, 5
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 77)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (capS, capT, *fwd, *bwd)]
    out = (torch.zeros(X * Y * Z, dtype=torch.uint8, device=dev), torch.zeros(X * Y * Z, dtype=torch.uint8, device=dev))
    B = Batch([(X, Y, Z)])
    try:
        B.bind_inputs(0, d[0].data_ptr(), d[1].data_ptr(), [t.data_ptr() for t in d[2:5]],
                      [t.data_ptr() for t in d[5:8]])
        B.bind_outputs(0, out[0].data_ptr(), out[1].data_ptr())
        B.enqueue(Policy())
        assert B.wait() == [f0]
        assert np.array_equal(out[0].cpu().numpy(), s0) and np.array_equal(out[1].cpu().numpy(), t0)
        d[2][7] = -3  # a negative n-link
        B.enqueue(Policy())
        with pytest.raises(_lib.CgcError) as e:
            B.wait()
        assert e.value.code == 1
        d[2][7] = 2 ** 30  # both directions of one link: more than int32 together
        d[5][7] = 2 ** 30
        B.enqueue(Policy())
        with pytest.raises(_lib.CgcError) as e:
            B.wait()
        assert e.value.code == 6
    finally:
        B.close()


@pytest.mark.parametrize("offset", [1, 3])
def test_outputs_at_unaligned_addresses(device_batch, offset):
    """Cut sets written to device buffers that start off a 4-byte boundary
    (byte stores instead of word stores), for instances whose voxel counts
    are not multiples of 4: the same bytes as the golden sets."""
    import torch
    B, vols, ins, outs, flows = device_batch
    dev = torch.device("cuda", 0)
    raw = [(torch.full((v.N + 8,), 7, dtype=torch.uint8, device=dev),
            torch.full((v.N + 8,), 7, dtype=torch.uint8, device=dev)) for v in vols]
    try:
        for i, r in enumerate(raw):
            B.bind_outputs(i, r[0].data_ptr() + offset, r[1].data_ptr() + offset)
        B.enqueue(Policy(), flows.data_ptr())
        fl = B.wait()
        shifted = [(r[0][offset:offset + v.N], r[1][offset:offset + v.N]) for r, v in zip(raw, vols)]
        _check(shifted, fl)
        for r, v in zip(raw, vols):  # nothing written around the outputs
            for buf in r:
                assert int(buf[:offset].ne(7).sum()) == 0
                assert int(buf[offset + v.N:].ne(7).sum()) == 0
    finally:
        for i, o in enumerate(outs):
            B.bind_outputs(i, o[0].data_ptr(), o[1].data_ptr())
    # the single-grid device output path
    v, d = vols[0], ins[0]  # 151 x 99 x 147: the voxel count is not a multiple of 4
    G = GridGraph(v.X, v.Y, v.Z)
    try:
        G.set_tweights_device(d[0].data_ptr(), d[1].data_ptr())
        for ax in range(3):
            G.set_nweights_device(ax, d[2 + ax].data_ptr())
        assert G.max_flow() == CASES[KEYS[0]]["flow"]
        buf = torch.full((v.N + 8,), 7, dtype=torch.uint8, device=dev)
        G.fill_segments_device(buf.data_ptr() + offset, 1, 0, SOURCE)
        assert sha(buf[offset:offset + v.N].cpu().numpy()) == CASES[KEYS[0]]["smin_sha256"]
        assert int(buf[:offset].ne(7).sum()) == 0 and int(buf[offset + v.N:].ne(7).sum()) == 0
        G.fill_segments_device(buf.data_ptr() + offset, 1, 0, SINK)
        assert sha(buf[offset:offset + v.N].cpu().numpy()) == CASES[KEYS[0]]["treach_sha256"]
    finally:
        G.close()


@pytest.mark.parametrize("policy", [None, Policy(local_pulses=2, region_relabels=4, sweeps_per_relabel=4, ctas_per_sm=4,
                                                 bfs_warp_min=8),
                                    Policy(exclusive=1, local_pulses=2, region_relabels=4, sweeps_per_relabel=4,
                                           ctas_per_sm=4, bfs_warp_min=8)])
def test_all_96_instances_match_the_oracle(policy):
    """The batched configuration itself: all 96 instances (extents 32..160)
    bound to one batch, the CUDA graph replayed twice, and every instance's
    flow and both cut sets compared with the oracle's golden answer."""
    import torch
    keys = [(4, i) for i in range(96)]
    vols = [volume.workload(*k) for k in keys]
    dev = torch.device("cuda", 0)
    ins = [[torch.from_numpy(a).to(dev) for a in v.arrays()] for v in vols]
    outs = [torch.full((2, v.N), 7, dtype=torch.uint8, device=dev) for v in vols]
    B = Batch([(v.X, v.Y, v.Z) for v in vols])
    try:
        for i, (d, o) in enumerate(zip(ins, outs)):
            B.bind_inputs(i, d[0].data_ptr(), d[1].data_ptr(), [t.data_ptr() for t in d[2:]])
            B.bind_outputs(i, o[0].data_ptr(), o[1].data_ptr())
        B.graph_create(policy)
        for rep in range(2):
            for o in outs:
                o.fill_(7)
            B.graph_launch()
            fl = B.wait()
            for i, k in enumerate(keys):
                c = CASES[k]
                assert fl[i] == c["flow"], k
                assert sha(outs[i][0].cpu().numpy()) == c["smin_sha256"], k
                assert sha(outs[i][1].cpu().numpy()) == c["treach_sha256"], k
    finally:
        B.close()
