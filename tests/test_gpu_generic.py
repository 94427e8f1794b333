"""Generic (non-grid) graphs on the GPU (cgc_graph_*): flow and both cut sets
against the CPU oracle's edge-list path, the reference's layered known
answers (unit_tests/graph_cut_test.cu:172-198) and the error contract."""
import numpy as np
import pytest

from cugip_b200 import _lib
from cugip_b200.graph_cut import SINK, SOURCE, GenericGraph, Graph, Policy
from oracle import oracle  # the checker

from tests import graphs

pytestmark = pytest.mark.gpu


def random_graph(n, m, seed, cmax=50, tmax=80, zero_frac=0.2, loops=0.0):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, n, m)
    b = rng.integers(0, n, m)
    if loops:
        sel = rng.random(m) < loops
        b[sel] = a[sel]
    cab = rng.integers(0, cmax, m)
    cba = rng.integers(0, cmax, m)
    cab[rng.random(m) < zero_frac] = 0
    cba[rng.random(m) < zero_frac] = 0
    capS = rng.integers(0, tmax, n)
    capT = rng.integers(0, tmax, n)
    capS[rng.random(n) < 0.5] = 0
    capT[rng.random(n) < 0.5] = 0
    return a, b, cab, cba, capS, capT


def solve(n, a, b, cab, cba, capS, capT, policy=None):
    with GenericGraph(n, a, b, cab, cba) as G:
        G.set_tweights(capS, capT)
        flow = G.max_flow(policy)
        return flow, G.fill_segments(mask=1, which=SOURCE), G.fill_segments(mask=1, which=SINK), G.stats()


POLICIES = [None, Policy(sweeps_per_relabel=1), Policy(sweeps_per_relabel=32)]


@pytest.mark.parametrize("policy", range(len(POLICIES)))
@pytest.mark.parametrize("n,m,seed", [(2, 1, 1), (10, 30, 2), (100, 300, 3), (1000, 2500, 4), (1000, 8000, 5),
                                      (5000, 12000, 6), (20000, 60000, 7), (3, 0, 8)])
def test_random_graphs_match_oracle(n, m, seed, policy):
    a, b, cab, cba, capS, capT = random_graph(n, m, seed)
    f0, s0, t0, _ = oracle.maxflow_edges(n, a, b, cab, cba, capS, capT)
    flow, smin, treach, st = solve(n, a, b, cab, cba, capS, capT, POLICIES[policy])
    assert flow == f0
    assert np.array_equal(smin, s0)
    assert np.array_equal(treach, t0)


@pytest.mark.parametrize("seed", range(4))
def test_long_paths_match_oracle(seed):
    """Sparse capacities over a long ring with chords: many BFS levels and pulses."""
    rng = np.random.default_rng(seed)
    n = 4000
    a = np.concatenate([np.arange(n), rng.integers(0, n, n // 10)])
    b = np.concatenate([(np.arange(n) + 1) % n, rng.integers(0, n, n // 10)])
    cab = rng.integers(1, 20, a.size)
    cba = rng.integers(0, 3, a.size)
    capS = np.zeros(n, np.int64)
    capT = np.zeros(n, np.int64)
    capS[rng.integers(0, n, 5)] = 1000
    capT[rng.integers(0, n, 5)] = 1000
    f0, s0, t0, _ = oracle.maxflow_edges(n, a, b, cab, cba, capS, capT)
    flow, smin, treach, _ = solve(n, a, b, cab, cba, capS, capT)
    assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


def test_self_loops_and_parallel_edges():
    a, b, cab, cba, capS, capT = random_graph(300, 2000, 11, loops=0.1)
    a = np.concatenate([a, a[:500]])  # parallel copies of 500 edges
    b = np.concatenate([b, b[:500]])
    cab = np.concatenate([cab, cab[:500]])
    cba = np.concatenate([cba, cba[:500]])
    f0, s0, t0, _ = oracle.maxflow_edges(300, a, b, cab, cba, capS, capT)
    flow, smin, treach, _ = solve(300, a, b, cab, cba, capS, capT)
    assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


@pytest.mark.parametrize("flip,expected", [(False, 1024 * 8), (True, 2 * 1024 * 8)])
def test_reference_layered_known_answers(flip, expected):
    n, a, b, f, g, s, t = graphs.layered(flip=flip)
    G = Graph()
    G.set_vertex_count(n)
    G.set_nweights(len(a), np.stack([a, b], 1), f, g)
    G.set_tweights(s, t)
    assert G.generic is not None
    assert G.max_flow() == expected
    f0, s0, t0, _ = oracle.maxflow_edges(n, a, b, f, g, s, t)
    assert f0 == expected
    assert np.array_equal(G.fill_segments(mask=1, which=SOURCE), s0)
    assert np.array_equal(G.fill_segments(mask=1, which=SINK), t0)


def test_grid_edge_lists_still_use_the_tile_engine():
    n, a, b, f, g, s, t = graphs.four_by_four()
    G = Graph()
    G.set_vertex_count(n)
    G.set_nweights(len(a), np.stack([a, b], 1), f, g)
    G.set_tweights(s, t)
    assert G.grid is not None and G.generic is None
    assert G.max_flow() == 4


def test_solving_again_gives_the_same_answer():
    a, b, cab, cba, capS, capT = random_graph(2000, 7000, 21)
    with GenericGraph(2000, a, b, cab, cba) as G:
        G.set_tweights(capS, capT)
        f1 = G.max_flow()
        s1 = G.fill_segments(mask=1, which=SOURCE)
        f2 = G.max_flow()
        assert f1 == f2 and np.array_equal(s1, G.fill_segments(mask=1, which=SOURCE))
        # new terminal capacities, same n-links
        G.set_tweights(capT, capS)
        f0, s0, t0, _ = oracle.maxflow_edges(2000, a, b, cab, cba, capT, capS)
        assert G.max_flow() == f0
        assert np.array_equal(G.fill_segments(mask=1, which=SINK), t0)


def test_terminal_only_vertices_and_isolated_vertices():
    n = 50
    capS = np.arange(n) % 7
    capT = (np.arange(n) * 3) % 5
    flow, smin, treach, _ = solve(n, [0], [1], [0], [0], capS, capT)
    f0, s0, t0, _ = oracle.maxflow_edges(n, [0], [1], [0], [0], capS, capT)
    assert flow == f0 == int(np.minimum(capS, capT).sum())
    assert np.array_equal(smin, s0) and np.array_equal(treach, t0)


def test_capacities_that_could_overflow_int32_are_refused():
    big = 2 ** 30 + 1
    with GenericGraph(3, [0, 1], [1, 2], [big, 1], [big, 1]) as G:  # one edge's two capacities exceed int32
        G.set_tweights([5, 0, 0], [0, 0, 5])
        with pytest.raises(_lib.CgcError) as e:
            G.max_flow()
        assert e.value.code == 6
    hub = np.zeros(3, np.int64)  # vertex 0 can receive 3 * 2^30: more than int32 excess
    with GenericGraph(4, hub, [1, 2, 3], [0, 0, 0], [2 ** 30] * 3) as G:
        G.set_tweights([0, 9, 9, 9], [9, 0, 0, 0])
        with pytest.raises(_lib.CgcError) as e:
            G.max_flow()
        assert e.value.code == 6
    with GenericGraph(2, [0], [1], [2 ** 30], [2 ** 30 - 1]) as G:  # at the limit: fine
        G.set_tweights([2 ** 30, 0], [0, 2 ** 30])
        assert G.max_flow() == 2 ** 30


def test_errors_are_loud():
    with pytest.raises(_lib.CgcError) as e:
        GenericGraph(4, [0, 5], [1, 2], [1, 1], [1, 1])
    assert e.value.code == 1
    with pytest.raises(_lib.CgcError) as e:
        GenericGraph(4, [0, 1], [1, 2], [1, -1], [1, 1])
    assert e.value.code == 1
    with GenericGraph(4, [0, 1], [1, 2], [1, 1], [1, 1]) as G:
        with pytest.raises(_lib.CgcError) as e:
            G.max_flow()
        assert e.value.code == 7  # terminal capacities missing
        with pytest.raises(_lib.CgcError) as e:
            G.fill_segments()
        assert e.value.code == 7
        with pytest.raises(_lib.CgcError) as e:
            G.set_tweights([1, 2, 3, -4], [0, 0, 0, 0])
        assert e.value.code == 1
