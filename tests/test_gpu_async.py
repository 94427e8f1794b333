"""The host path in two halves (cgc_grid_maxflow_async / cgc_grid_wait): two
grids on their own streams, one uploading while the other solves, must give
the oracle's exact flows and cut sets, in any interleaving of the calls; the
calls that read results are refused while a solve is queued."""
import json
import os

import numpy as np
import pytest

from cugip_b200 import _lib, volume
from cugip_b200.graph_cut import SINK, SOURCE, Batch, GridGraph, Policy
from tests import graphs
from tests.gpu_helpers import sha

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")))
CASES = {(c["workload"], c["index"]): c for c in GOLDEN["cases"]}


def _set(g, v):
    g.set_tweights(v.capS, v.capT)
    for ax in range(3):
        g.set_nweights(ax, v.n[ax])


def _check(g, key):
    c = CASES[key]
    assert g.flow == c["flow"], key
    assert sha(g.fill_segments(mask=1, which=SOURCE)) == c["smin_sha256"], key
    assert sha(g.fill_segments(mask=1, which=SINK)) == c["treach_sha256"], key


@pytest.mark.parametrize("policy", [None, Policy(ctas_per_sm=3), Policy(persistent=-1)])
def test_two_grids_pipelined(policy):
    """Each step uploads grid i while grid i-1 solves, then reads grid i-1's
    results: the order of the bench's end-to-end loop."""
    import torch
    keys = [(4, i) for i in range(6)]
    vols = [volume.workload(*k) for k in keys]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    grids = {}
    try:
        prev = None
        for i, (k, v) in enumerate(zip(keys, vols)):
            g = GridGraph(v.X, v.Y, v.Z, stream=streams[i % 2].cuda_stream)
            grids[k] = g
            _set(g, v)
            g.max_flow_async(policy)
            if prev is not None:
                pk, pg = prev
                pg.wait()
                _check(pg, pk)
            prev = (k, g)
        prev[1].wait()
        _check(prev[1], prev[0])
    finally:
        for g in grids.values():
            g.close()


def test_reuse_one_grid_with_uploads_during_the_solve():
    """The next capacities may be set while the previous solve is queued: the
    copies wait until the queued upload kernel has read the planes."""
    v = volume.workload(4, 3)
    w = volume.workload(4, 3)  # the same instance, scaled by 2 for the second solve
    g = GridGraph(v.X, v.Y, v.Z)
    try:
        _set(g, v)
        g.max_flow_async()
        # scaled capacities (flow doubles, cut sets stay) uploaded while the first solve runs
        g.set_tweights(2 * w.capS, 2 * w.capT)
        for ax in range(3):
            g.set_nweights(ax, 2 * w.n[ax])
        assert g.wait() == CASES[(4, 3)]["flow"]
        _check(g, (4, 3))
        assert g.max_flow() == 2 * CASES[(4, 3)]["flow"]
        assert sha(g.fill_segments(mask=1, which=SOURCE)) == CASES[(4, 3)]["smin_sha256"]
        assert sha(g.fill_segments(mask=1, which=SINK)) == CASES[(4, 3)]["treach_sha256"]
    finally:
        g.close()


def test_results_are_refused_while_a_solve_is_queued():
    v = volume.workload(1)
    g = GridGraph(v.X, v.Y, v.Z)
    try:
        with pytest.raises(_lib.CgcError) as e:
            g.wait()
        assert e.value.code == 7
        _set(g, v)
        g.max_flow_async()
        for call in (lambda: g.fill_segments(), lambda: g.residuals(), lambda: g.max_flow_async(),
                     lambda: g.max_flow()):
            with pytest.raises(_lib.CgcError) as e:
                call()
            assert e.value.code == 7
        assert g.wait() == CASES[(1, 0)]["flow"]
        _check(g, (1, 0))
    finally:
        g.close()


@pytest.mark.parametrize("mask,bg", [(255, 0), (1, 0), (3, 200), (0, 9)])
def test_mask_and_background_values(mask, bg):
    """Any mask / background pair, to host and to device memory (the reference's
    fill_segments defaults to 255 / 0, graph_cut.hpp:318-333)."""
    import torch
    from oracle import oracle  # the checker
    X, Y, Z = 37, 21, 11  # odd voxel count: the 16-byte path and its tail
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 31)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    g = GridGraph(X, Y, Z)
    try:
        g.set_tweights(capS, capT)
        for ax in range(3):
            g.set_nweights(ax, fwd[ax], bwd[ax])
        assert g.max_flow() == f0
        for which, ref in ((SOURCE, s0), (SINK, t0)):
            want = np.where(ref.astype(bool), mask, bg).astype(np.uint8)
            assert np.array_equal(g.fill_segments(mask=mask, background=bg, which=which), want)
            d = torch.full((X * Y * Z + 16,), 77, dtype=torch.uint8, device="cuda")
            for off in (0, 1):
                g.fill_segments_device(d.data_ptr() + off, mask, bg, which)
                assert np.array_equal(d[off:off + X * Y * Z].cpu().numpy(), want)
    finally:
        g.close()


def test_host_batch_uses_the_same_upload():
    """Host setters on a batch of several instances: the fused upload reads a
    device table of the instances' input planes."""
    keys = [(4, i) for i in range(8, 14)]
    vols = [volume.workload(*k) for k in keys]
    B = Batch([(v.X, v.Y, v.Z) for v in vols])
    try:
        for rep in range(2):
            for i, v in enumerate(vols):
                B.set_tweights(i, v.capS, v.capT)
                for ax in range(3):
                    B.set_nweights(i, ax, v.n[ax])
            fl = B.max_flow(Policy(ctas_per_sm=4, bfs_warp_min=8) if rep else None)
            for i, k in enumerate(keys):
                assert fl[i] == CASES[k]["flow"], k
                assert sha(B.fill_segments(i, mask=1, which=SOURCE)) == CASES[k]["smin_sha256"], k
                assert sha(B.fill_segments(i, mask=1, which=SINK)) == CASES[k]["treach_sha256"], k
    finally:
        B.close()
