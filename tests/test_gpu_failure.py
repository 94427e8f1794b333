"""Failure detection on the GPU, in the safe forms: every device-side wait of
the solver is bounded (cgc_options.wait_limit_us), and a wait that runs out
ends the solve with CGC_ERR_TIMEOUT instead of hanging; a solve that reaches
max_sweeps ends with CGC_ERR_NOT_CONVERGED.  Nothing here faults, traps or
hangs a GPU: the short limit only makes a grid barrier give up early, the
kernel returns, the host reads the status, and the same handle then solves
exactly.

The reference's grid barrier (cub::GridBarrier in
include/cugip/advanced_operations/detail/graph_cut_relabeling.hpp:717-751)
spins without a limit, and its host loop has no iteration cap
(detail/graph_cut_implementation.hpp:152-194)."""
import json
import os

import numpy as np
import pytest

from cugip_b200 import _lib, volume
from cugip_b200.graph_cut import SINK, SOURCE, Batch, GenericGraph, GridGraph, Policy
from tests import graphs
from tests.gpu_helpers import sha

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")))
CASES = {(c["workload"], c["index"]): c for c in GOLDEN["cases"]}
TIMEOUT, NOT_CONVERGED = 4, 5

# a 1 us bound: some CTA of the persistent launch waits longer than that at a
# grid barrier in every solve (a tile visit alone takes several us)
SHORT_WAIT = dict(wait_limit_us=1)


def _upload(g, v):
    g.set_tweights(v.capS, v.capT)
    for ax in range(3):
        g.set_nweights(ax, v.n[ax])


def _check_grid(g, key):
    c = CASES[key]
    assert sha(g.fill_segments(mask=1, which=SOURCE)) == c["smin_sha256"]
    assert sha(g.fill_segments(mask=1, which=SINK)) == c["treach_sha256"]


@pytest.mark.parametrize("ctas", [2, 3, 4])
def test_grid_wait_limit_times_out_then_recovers(ctas):
    v = volume.workload(1)
    g = GridGraph(v.X, v.Y, v.Z)
    try:
        _upload(g, v)
        with pytest.raises(_lib.CgcError) as e:
            g.max_flow(Policy(ctas_per_sm=ctas, **SHORT_WAIT))
        assert e.value.code == TIMEOUT
        # the planes hold a partial preflow now: solving again needs new capacities
        with pytest.raises(_lib.CgcError) as e:
            g.max_flow()
        assert e.value.code == 7
        _upload(g, v)
        assert g.max_flow(Policy(ctas_per_sm=ctas)) == CASES[(1, 0)]["flow"]
        _check_grid(g, (1, 0))
    finally:
        g.close()


@pytest.mark.parametrize("policy", [Policy(max_sweeps=1), Policy(max_sweeps=1, persistent=-1),
                                    Policy(max_sweeps=1, ctas_per_sm=4, bfs_warp_min=8)])
def test_grid_max_sweeps_reports_not_converged_then_recovers(policy):
    v = volume.workload(1)
    g = GridGraph(v.X, v.Y, v.Z)
    try:
        _upload(g, v)
        with pytest.raises(_lib.CgcError) as e:
            g.max_flow(policy)
        assert e.value.code == NOT_CONVERGED
        _upload(g, v)
        assert g.max_flow() == CASES[(1, 0)]["flow"]
        _check_grid(g, (1, 0))
    finally:
        g.close()


def test_generic_graph_wait_limit_and_pulse_cap():
    from oracle import oracle  # the checker
    n, a, b, f, w, s, t = graphs.layered(layers=12, size=64, nbrs=4)
    f0, s0, t0, _ = oracle.maxflow_edges(n, a, b, f, w, s, t)
    with GenericGraph(n, a, b, f, w) as g:
        g.set_tweights(s, t)
        with pytest.raises(_lib.CgcError) as e:
            g.max_flow(Policy(**SHORT_WAIT))
        assert e.value.code == TIMEOUT
        with pytest.raises(_lib.CgcError) as e:
            g.max_flow(Policy(max_sweeps=1, sweeps_per_relabel=1))
        assert e.value.code == NOT_CONVERGED
        # the generic engine keeps the capacities: it solves again directly
        assert g.max_flow() == f0
        assert np.array_equal(g.fill_segments(mask=1, which=SOURCE), s0)
        assert np.array_equal(g.fill_segments(mask=1, which=SINK), t0)


def test_batch_wait_limit_and_max_sweeps_then_recovers():
    """Device-resident batch: the error comes back through cgc_batch_wait, for
    a direct enqueue and for a CUDA-graph replay, and the next enqueue (which
    re-reads the bound inputs) is exact again."""
    import torch
    keys = [(4, i) for i in range(4)]
    vols = [volume.workload(*k) for k in keys]
    dev = torch.device("cuda", 0)
    ins = [[torch.from_numpy(x).to(dev) for x in v.arrays()] for v in vols]
    outs = [torch.zeros((2, v.N), dtype=torch.uint8, device=dev) for v in vols]
    B = Batch([(v.X, v.Y, v.Z) for v in vols])
    try:
        for i, (d, o) in enumerate(zip(ins, outs)):
            B.bind_inputs(i, d[0].data_ptr(), d[1].data_ptr(), [x.data_ptr() for x in d[2:]])
            B.bind_outputs(i, o[0].data_ptr(), o[1].data_ptr())
        for bad, code in ((Policy(**SHORT_WAIT), TIMEOUT), (Policy(ctas_per_sm=4, **SHORT_WAIT), TIMEOUT),
                          (Policy(max_sweeps=1), NOT_CONVERGED)):
            B.enqueue(bad)
            with pytest.raises(_lib.CgcError) as e:
                B.wait()
            assert e.value.code == code
            B.graph_create(bad)
            B.graph_launch()
            with pytest.raises(_lib.CgcError) as e:
                B.wait()
            assert e.value.code == code
            B.enqueue(Policy())
            fl = B.wait()
            for i, k in enumerate(keys):
                assert fl[i] == CASES[k]["flow"]
                assert sha(outs[i][0].cpu().numpy()) == CASES[k]["smin_sha256"]
                assert sha(outs[i][1].cpu().numpy()) == CASES[k]["treach_sha256"]
    finally:
        B.close()
