"""The allocation-free entry point (cgc_grid_maxflow_noalloc) against the
ordinary one (cgc_grid_maxflow).

cgc_grid_maxflow_noalloc exists for callers that may not allocate device
memory themselves through a library: processes whose device memory belongs to
another allocator, and real-time loops that cannot take the synchronisation of
cudaMalloc / cudaFree.  Its working state is a static device array of fixed
size, shared by every call.  These tests call it twice in a row on the same
inputs (the second call starts from whatever the first left in the array) and
compare flow and both cut masks with the ordinary entry point: the results
must be identical (the engine is exact, so the tolerance is zero).

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from cugip_b200 import _lib, volume
from cugip_b200.graph_cut import SINK, SOURCE, GridGraph
from tests import graphs

pytestmark = pytest.mark.gpu


def _reference_solve(X, Y, Z, capS, capT, fwd, bwd):
    g = GridGraph(X, Y, Z)
    try:
        g.set_tweights(capS, capT)
        for ax in range(3):
            g.set_nweights(ax, fwd[ax], bwd[ax])
        flow = g.max_flow()
        return flow, g.fill_segments(mask=1, which=SOURCE), g.fill_segments(mask=1, which=SINK)
    finally:
        g.close()


def _noalloc_solve(X, Y, Z, capS, capT, fwd, bwd, opts=None, stream=None, outputs=(True, True), rc_only=False):
    """One call of the entry point on device copies of the inputs; an axis whose
    fwd entry is None is passed as a NULL plane pair (zero capacity)."""
    import torch
    dev = torch.device("cuda", 0)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(dev)
    d_s, d_t = d(capS), d(capT)
    d_f = [None if a is None else d(a) for a in fwd]
    d_b = [None if a is None else d(a) for a in bwd]
    N = X * Y * Z
    out_s = torch.full((N,), 7, dtype=torch.uint8, device=dev)
    out_t = torch.full((N,), 7, dtype=torch.uint8, device=dev)
    fp = (C.c_void_p * 3)(*[None if t is None else t.data_ptr() for t in d_f])
    bp = (C.c_void_p * 3)(*[None if t is None else t.data_ptr() for t in d_b])
    flow = C.c_int64(-1)
    torch.cuda.synchronize()
    rc = _lib.load().cgc_grid_maxflow_noalloc(X, Y, Z, d_s.data_ptr(), d_t.data_ptr(), fp, bp,
                                              C.byref(opts) if opts is not None else None,
                                              C.c_void_p(stream.cuda_stream) if stream is not None else None,
                                              C.byref(flow), out_s.data_ptr() if outputs[0] else None,
                                              out_t.data_ptr() if outputs[1] else None)
    if rc_only:
        return rc
    _lib.check(rc)
    return int(flow.value), out_s.cpu().numpy(), out_t.cpu().numpy()


def _cases():
    v = volume.workload(1)  # 64^3: exactly the largest grid the static scratch holds
    yield "workload1_64cubed", (v.X, v.Y, v.Z, v.capS, v.capT, v.n, v.n)
    X, Y, Z = 40, 24, 17
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 4242)
    yield "random_40x24x17", (X, Y, Z, capS, capT, fwd, bwd)


@pytest.mark.parametrize("name,case", list(_cases()))
def test_noalloc_matches_the_allocating_entry_point_twice(name, case):
    import torch
    _lib.check(_lib.load().cgc_init(0))
    ref = _reference_solve(*case)
    for call in range(2):
        flow, smin, treach = _noalloc_solve(*case)
        assert flow == ref[0], (name, call)
        assert np.array_equal(smin, ref[1]), (name, call)
        assert np.array_equal(treach, ref[2]), (name, call)
    torch.cuda.synchronize()


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    _lib.check(_lib.load().cgc_init(0))
    flow = C.c_int64(0)
    zero = (C.c_void_p * 3)()
    # 65 rounds up to 72: 72*64*64 padded voxels exceed CGC_NOALLOC_MAX_VOXELS
    rc = _lib.load().cgc_grid_maxflow_noalloc(65, 64, 64, C.c_void_p(16), C.c_void_p(16), zero, zero, None, None,
                                              C.byref(flow), None, None)
    assert rc == 1  # CGC_ERR_ARG, nothing launched
    assert b"static scratch" in _lib.load().cgc_last_error()


def test_noalloc_matches_the_oracle():
    from oracle import oracle  # the checker
    _lib.check(_lib.load().cgc_init(0))
    X, Y, Z = 33, 17, 9
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 99)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    flow, smin, treach = _noalloc_solve(X, Y, Z, capS, capT, fwd, bwd)
    assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


def test_noalloc_null_axis_and_one_output_at_a_time():
    """A NULL axis has zero capacity (like an axis never set on a GridGraph),
    and each cut set can be requested alone; the other buffer is left as is."""
    from oracle import oracle  # the checker
    _lib.check(_lib.load().cgc_init(0))
    X, Y, Z = 24, 20, 12
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 7)
    z = np.zeros(X * Y * Z, np.int32)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, [fwd[0], z, fwd[2]], [bwd[0], z, bwd[2]])
    nf, nb = [fwd[0], None, fwd[2]], [bwd[0], None, bwd[2]]
    flow, smin, untouched = _noalloc_solve(X, Y, Z, capS, capT, nf, nb, outputs=(True, False))
    assert flow == f0 and np.array_equal(smin, s0) and (untouched == 7).all()
    flow, untouched, treach = _noalloc_solve(X, Y, Z, capS, capT, nf, nb, outputs=(False, True))
    assert flow == f0 and np.array_equal(treach, t0) and (untouched == 7).all()


def test_noalloc_options_and_side_stream():
    import torch
    _lib.check(_lib.load().cgc_init(0))
    v = volume.workload(1)
    case = (v.X, v.Y, v.Z, v.capS, v.capT, v.n, v.n)
    ref = _reference_solve(*case)
    side = torch.cuda.Stream()
    for opts in (_lib.options(local_pulses=2, region_relabels=4, sweeps_per_relabel=3),
                 _lib.options(local_pulses=8, region_relabels=-1, stall_sweeps=2)):
        flow, smin, treach = _noalloc_solve(*case, opts=opts, stream=side)
        assert flow == ref[0] and np.array_equal(smin, ref[1]) and np.array_equal(treach, ref[2])


def test_noalloc_not_converged_then_exact_again():
    """max_sweeps reached: CGC_ERR_NOT_CONVERGED; the next call starts from
    what that one left in the shared array and must still be exact."""
    _lib.check(_lib.load().cgc_init(0))
    v = volume.workload(1)
    case = (v.X, v.Y, v.Z, v.capS, v.capT, v.n, v.n)
    ref = _reference_solve(*case)
    assert _noalloc_solve(*case, opts=_lib.options(max_sweeps=1), rc_only=True) == 5
    flow, smin, treach = _noalloc_solve(*case)
    assert flow == ref[0] and np.array_equal(smin, ref[1]) and np.array_equal(treach, ref[2])
