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


def _noalloc_solve(X, Y, Z, capS, capT, fwd, bwd):
    import torch
    dev = torch.device("cuda", 0)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(dev)
    d_s, d_t = d(capS), d(capT)
    d_f = [d(a) for a in fwd]
    d_b = [d(a) for a in bwd]
    N = X * Y * Z
    out_s = torch.full((N,), 7, dtype=torch.uint8, device=dev)
    out_t = torch.full((N,), 7, dtype=torch.uint8, device=dev)
    fp = (C.c_void_p * 3)(*[t.data_ptr() for t in d_f])
    bp = (C.c_void_p * 3)(*[t.data_ptr() for t in d_b])
    flow = C.c_int64(-1)
    torch.cuda.synchronize()
    rc = _lib.load().cgc_grid_maxflow_noalloc(X, Y, Z, d_s.data_ptr(), d_t.data_ptr(), fp, bp, None, None,
                                              C.byref(flow), out_s.data_ptr(), out_t.data_ptr())
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
