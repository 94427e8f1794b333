"""Helpers of the GPU parity tests: solve through the C ABI and certify."""
from __future__ import annotations

import hashlib

import numpy as np

from cugip_b200.graph_cut import SINK, SOURCE, GridGraph, Policy


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def solve(X, Y, Z, capS, capT, fwd, bwd=None, policy=None, residuals=False):
    """Returns (flow, smin uint8, treach uint8, stats[, residuals]) from the GPU."""
    g = GridGraph(X, Y, Z)
    try:
        g.set_tweights(capS, capT)
        for ax in range(3):
            g.set_nweights(ax, fwd[ax], None if bwd is None else bwd[ax])
        flow = g.max_flow(policy)
        smin = g.fill_segments(mask=1, background=0, which=SOURCE)
        treach = g.fill_segments(mask=1, background=0, which=SINK)
        out = [flow, smin, treach, g.stats()]
        if residuals:
            out.append(g.residuals())
        return tuple(out)
    finally:
        g.close()


def certify(X, Y, Z, capS, capT, fwd, bwd, flow, res, smin, treach):
    """Exact optimality certificate from the final residual graph:
    a feasible preflow of value `flow` and cuts of capacity `flow`."""
    from oracle.oracle import cut_capacity_grid  # the checker
    bwd = fwd if bwd is None else bwd
    N = X * Y * Z
    shape = (Z, Y, X)
    r = res["r"].astype(np.int64).reshape(6, *shape)
    rT = res["resT"].astype(np.int64).reshape(shape)
    ex = res["excess"].astype(np.int64).reshape(shape)
    cs = np.asarray(capS, np.int64).reshape(shape)
    ct = np.asarray(capT, np.int64).reshape(shape)
    m = np.minimum(cs, ct)
    assert (r >= 0).all() and (rT >= 0).all() and (ex >= 0).all()
    assert (rT <= ct - m).all()
    net_out = np.zeros(shape, np.int64)
    for ax, axnp in ((0, 2), (1, 1), (2, 0)):
        f = np.asarray(fwd[ax], np.int64).reshape(shape)
        b = np.asarray(bwd[ax], np.int64).reshape(shape)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axnp] = slice(0, -1)
        hi[axnp] = slice(1, None)
        lo, hi = tuple(lo), tuple(hi)
        rp, rm = r[2 * ax], r[2 * ax + 1]
        # residuals of an edge pair add up to its two capacities
        assert np.array_equal(rp[lo] + rm[hi], f[lo] + b[lo])
        # edges leaving the grid carry nothing
        edge = [slice(None)] * 3
        edge[axnp] = -1
        assert (rp[tuple(edge)] == 0).all()
        edge[axnp] = 0
        assert (rm[tuple(edge)] == 0).all()
        flow_lo_hi = f[lo] - rp[lo]  # net flow lo -> hi
        net_out[lo] += flow_lo_hi
        net_out[hi] -= flow_lo_hi
    # conservation: excess = source inflow - n-link outflow - sink outflow
    sink_out = m + (ct - m - rT)
    assert np.array_equal(ex, cs - net_out - sink_out)
    assert int(sink_out.sum()) == flow
    assert cut_capacity_grid(X, Y, Z, capS, capT, fwd, bwd, smin) == flow
    assert cut_capacity_grid(X, Y, Z, capS, capT, fwd, bwd, ~treach.astype(bool)) == flow
    # excess only where the sink is unreachable
    assert not (ex.reshape(-1) > 0)[treach.astype(bool)].any()
