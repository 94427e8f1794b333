"""The CPU oracle pinned against the reference's known answers and against
brute force, before any GPU result is compared with it."""
import itertools

import numpy as np
import pytest

from oracle import oracle
from tests import graphs


@pytest.mark.parametrize("algo", [oracle.BK, oracle.DINIC])
def test_four_by_four_known_answer(algo):
    n, a, b, f, g, s, t = graphs.four_by_four()
    flow, smin, treach, _ = oracle.maxflow_edges(n, a, b, f, g, s, t, algo=algo)
    assert flow == 4
    # the cut is the row 1 -> row 2 layer: rows 0,1 on the source side
    assert smin.tolist() == [1] * 8 + [0] * 8
    assert treach.tolist() == [0] * 8 + [1] * 8


@pytest.mark.parametrize("flip,expected", [(False, 1024 * 8), (True, 2 * 1024 * 8)])
@pytest.mark.parametrize("algo", [oracle.BK, oracle.DINIC])
def test_layered_known_answer(algo, flip, expected):
    n, a, b, f, g, s, t = graphs.layered(flip=flip)
    flow, smin, treach, _ = oracle.maxflow_edges(n, a, b, f, g, s, t, algo=algo)
    assert flow == expected


def brute_force(n, a, b, f, g, s, t):
    """All minimum cuts of a tiny graph by enumeration: (value, intersection of
    the min-cut source sides, union of the min-cut source sides)."""
    best, inter, union = None, None, None
    for bits in itertools.product([0, 1], repeat=n):
        S = np.array(bits, bool)
        val = int(t[S].sum() + s[~S].sum())
        val += int(f[S[a] & ~S[b]].sum() + g[S[b] & ~S[a]].sum())
        if best is None or val < best:
            best, inter, union = val, S.copy(), S.copy()
        elif val == best:
            inter &= S
            union |= S
    return best, inter, union


@pytest.mark.parametrize("seed", range(40))
def test_random_small_graphs_brute_force(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 11))
    m = int(rng.integers(1, 3 * n))
    a = rng.integers(0, n, m)
    b = (a + rng.integers(1, n, m)) % n
    cap = lambda k: np.where(rng.random(k) < 0.3, 0, rng.integers(0, 8, k))
    f, g, s, t = cap(m), cap(m), cap(n), cap(n)
    best, inter, union = brute_force(n, a, b, f, g, s, t)
    for algo in (oracle.BK, oracle.DINIC):
        flow, smin, treach, _ = oracle.maxflow_edges(n, a, b, f, g, s, t, algo=algo)
        assert flow == best
        # minimal source side = intersection of all min-cut source sides;
        # the sink-reachable set is the complement of their union
        assert smin.astype(bool).tolist() == inter.tolist()
        assert (~treach.astype(bool)).tolist() == union.tolist()


@pytest.mark.parametrize("dims,seed", [((7, 5, 3), 1), ((16, 16, 4), 2), ((9, 1, 1), 3), ((12, 10, 1), 4),
                                       ((20, 17, 13), 5)])
def test_bk_matches_dinic_on_random_grids(dims, seed):
    X, Y, Z = dims
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, seed)
    r1 = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd, algo=oracle.BK)
    r2 = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd, algo=oracle.DINIC)
    assert r1[0] == r2[0]
    assert np.array_equal(r1[1], r2[1]) and np.array_equal(r1[2], r2[2])
    # the cut through the minimal source side has the flow's capacity
    assert oracle.cut_capacity_grid(X, Y, Z, capS, capT, fwd, bwd, r1[1]) == r1[0]
    assert oracle.cut_capacity_grid(X, Y, Z, capS, capT, fwd, bwd, ~r1[2].astype(bool)) == r1[0]


def test_grid_builder_matches_edge_builder():
    X, Y, Z = 11, 6, 5
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 9)
    a, b, f, g = graphs.grid_edges(X, Y, Z, fwd, bwd)
    r1 = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    r2 = oracle.maxflow_edges(X * Y * Z, a, b, f, g, capS, capT, algo=oracle.DINIC)
    assert r1[0] == r2[0]
    assert np.array_equal(r1[1], r2[1]) and np.array_equal(r1[2], r2[2])
