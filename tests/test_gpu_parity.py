"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle and the
golden fixtures -- exact flow value and bit-identical cut sets."""
import json
import os

import numpy as np
import pytest

from cugip_b200 import _lib, volume
from cugip_b200.graph_cut import SINK, SOURCE, Batch, Graph, GridGraph, Policy
from oracle import oracle
from tests import graphs
from tests.gpu_helpers import certify, sha, solve

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")))
CASES = {(c["workload"], c["index"]): c for c in GOLDEN["cases"]}

POLICIES = {
    "default": None,
    "host_loop": Policy(persistent=-1),
    "L1_K1": Policy(local_pulses=1, sweeps_per_relabel=1),
    "L4_K2": Policy(local_pulses=4, sweeps_per_relabel=2),
    "L32_K32": Policy(local_pulses=32, sweeps_per_relabel=32),
    "host_L2": Policy(local_pulses=2, sweeps_per_relabel=3, persistent=-1),
    "no_region": Policy(region_relabels=-1),
    "R3_L2": Policy(local_pulses=2, region_relabels=3, sweeps_per_relabel=2),
    "host_R2": Policy(region_relabels=2, persistent=-1),
    "stall1_K64": Policy(stall_sweeps=1, sweeps_per_relabel=64),
    "stall3_L2": Policy(stall_sweeps=3, local_pulses=2, sweeps_per_relabel=16),
    "cta4_R4": Policy(ctas_per_sm=4, region_relabels=4),
    "bfsw_all": Policy(ctas_per_sm=3, bfs_warp_min=1),
    "bfsw8_cta4": Policy(ctas_per_sm=4, region_relabels=4, bfs_warp_min=8),
    "cta3_L2_R4": Policy(ctas_per_sm=3, local_pulses=2, region_relabels=4, sweeps_per_relabel=2),
    "cta3_L1_K1": Policy(ctas_per_sm=3, local_pulses=1, sweeps_per_relabel=1),
    "cta4_no_region": Policy(ctas_per_sm=4, region_relabels=-1, local_pulses=8),
    "cta3_stall": Policy(ctas_per_sm=3, stall_sweeps=1, sweeps_per_relabel=64),
    "cta4_bfsw_K2": Policy(ctas_per_sm=4, bfs_warp_min=1, local_pulses=2, sweeps_per_relabel=2),
    "excl": Policy(exclusive=1),
    "excl_cta3_L1_K1": Policy(exclusive=1, ctas_per_sm=3, local_pulses=1, sweeps_per_relabel=1),
    "excl_cta4_bfsw": Policy(exclusive=1, ctas_per_sm=4, region_relabels=4, bfs_warp_min=8),
    "excl_stall": Policy(exclusive=1, stall_sweeps=1, sweeps_per_relabel=64),
    # every global relabel a full BFS from the sink (the default re-checks
    # only what the last sweep cycle touched)
    "full_relabel": Policy(relabel=1),
    "full_cta4_bfsw": Policy(relabel=1, ctas_per_sm=4, region_relabels=4, bfs_warp_min=8),
    "full_excl_L1_K1": Policy(relabel=1, exclusive=1, local_pulses=1, sweeps_per_relabel=1),
}


def test_reference_four_by_four_through_graph_api():
    n, a, b, f, g, s, t = graphs.four_by_four()
    G = Graph()
    G.set_vertex_count(n)
    G.set_tweights(s.astype(np.float32), t.astype(np.float32))  # reference tests pass float weights
    G.set_nweights(len(a), np.stack([a, b], 1), f.astype(np.float32), g.astype(np.float32))
    assert G.max_flow() == 4
    out = np.zeros(16, np.uint8)
    G.fill_segments(out)  # default mask 255 / background 0: sink-reachable vertices
    assert out.tolist() == [0] * 8 + [255] * 8
    assert G.fill_segments(mask=1, which=SOURCE).tolist() == [1] * 8 + [0] * 8


def test_layered_reference_graph_goes_to_the_generic_engine():
    n, a, b, f, g, s, t = graphs.layered(layers=6, size=32, nbrs=4)
    G = Graph()
    G.set_vertex_count(n)
    G.set_nweights(len(a), np.stack([a, b], 1), f, g)
    G.set_tweights(s, t)
    assert G.generic is not None and G.grid is None
    f0, s0, t0, _ = oracle.maxflow_edges(n, a, b, f, g, s, t)
    assert G.max_flow() == f0
    assert np.array_equal(G.fill_segments(mask=1, which=SOURCE), s0)
    assert np.array_equal(G.fill_segments(mask=1, which=SINK), t0)


@pytest.mark.parametrize("policy", list(POLICIES))
@pytest.mark.parametrize("dims,seed", [((8, 8, 8), 1), ((7, 5, 3), 2), ((16, 16, 4), 3), ((9, 1, 1), 4),
                                       ((33, 17, 9), 5), ((64, 8, 8), 6), ((20, 20, 20), 7), ((1, 1, 1), 8),
                                       ((40, 3, 17), 9)])
def test_random_grids_match_oracle(dims, seed, policy):
    X, Y, Z = dims
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, seed)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    flow, smin, treach, st, res = solve(X, Y, Z, capS, capT, fwd, bwd, POLICIES[policy], residuals=True)
    assert flow == f0
    assert np.array_equal(smin, s0)
    assert np.array_equal(treach, t0)
    certify(X, Y, Z, capS, capT, fwd, bwd, flow, res, smin, treach)


@pytest.mark.parametrize("seed", range(6))
def test_long_paths_match_oracle(seed):
    """Sparse capacities: long thin augmenting paths (many BFS rounds, many sweeps)."""
    X, Y, Z = 48, 40, 24
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 100 + seed, tmax=30, nmax=20, zero_frac=0.9)
    for f in fwd + bwd:
        f[np.random.default_rng(seed).random(f.size) < 0.4] = 0
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    for pol in (None, Policy(persistent=-1), POLICIES["cta3_L2_R4"], POLICIES["cta4_no_region"], POLICIES["excl"],
                POLICIES["excl_cta3_L1_K1"]):
        flow, smin, treach, _ = solve(X, Y, Z, capS, capT, fwd, bwd, pol)
        assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


@pytest.mark.parametrize("policy", ["default", "cta4_R4", "bfsw_all", "bfsw8_cta4", "cta3_L2_R4", "excl",
                                    "excl_cta4_bfsw", "full_relabel"])
@pytest.mark.parametrize("key", [k for k in CASES if k[0] in (1, 5) or (k[0] == 4 and k[1] < 8)])
def test_golden_workloads(key, policy):
    c = CASES[key]
    v = volume.workload(*key)
    assert sha(*v.arrays()) == c["volume_sha256"]
    flow, smin, treach, st = solve(v.X, v.Y, v.Z, v.capS, v.capT, v.n, None, POLICIES[policy])
    assert flow == c["flow"]
    assert sha(smin) == c["smin_sha256"]
    assert sha(treach) == c["treach_sha256"]


@pytest.mark.parametrize("policy", ["default", "bfsw8_cta4", "cta3_L2_R4", "excl", "excl_cta4_bfsw",
                                    "full_cta4_bfsw"])
@pytest.mark.parametrize("key", [(2, 0), (3, 0)])
def test_full_size_workloads_with_certificate(key, policy):
    c = CASES[key]
    v = volume.workload(*key)
    flow, smin, treach, st, res = solve(v.X, v.Y, v.Z, v.capS, v.capT, v.n, None, POLICIES[policy], residuals=True)
    assert flow == c["flow"]
    assert sha(smin) == c["smin_sha256"] and sha(treach) == c["treach_sha256"]
    certify(v.X, v.Y, v.Z, v.capS, v.capT, v.n, None, flow, res, smin, treach)


def _solve_with_labels(v, policy):
    g = GridGraph(v.X, v.Y, v.Z)
    try:
        g.set_tweights(v.capS, v.capT)
        for ax in range(3):
            g.set_nweights(ax, v.n[ax])
        flow = g.max_flow(policy)
        return flow, g.labels(), g.stats(), g.fill_segments(mask=1, background=0, which=SOURCE)
    finally:
        g.close()


@pytest.mark.parametrize("base", ["default", "L1_K1", "cta3_L2_R4", "bfsw8_cta4", "stall3_L2", "excl",
                                  "excl_cta3_L1_K1"])
@pytest.mark.parametrize("key", [(1, 0), (4, 3), (4, 6), (5, 0), (2, 0), (3, 0)])
def test_incremental_relabel_equals_full_bfs(key, base):
    """The incremental global relabel (invalidation from the tiles a sweep
    cycle queued, then tile Bellman-Ford from the dropped voxels) must leave
    the full BFS's labels bit for bit.  Every later step depends only on the
    labels, so both solves take the same sweeps, tile visits and pulses and end
    with the same labels, flow and cuts."""
    c = CASES[key]
    v = volume.workload(*key)
    pol = POLICIES[base] or Policy()
    full = _solve_with_labels(v, pol.with_(relabel=1))
    inc = _solve_with_labels(v, pol.with_(relabel=2))
    assert full[0] == inc[0] == c["flow"]
    assert np.array_equal(full[1], inc[1])
    for k in ("sweeps", "global_relabels", "tiles_swept", "pulses"):
        assert full[2][k] == inc[2][k], k
    assert full[2]["tiles_checked"] == 0
    if inc[2]["global_relabels"] > 1:
        assert inc[2]["tiles_checked"] > 0
    assert sha(inc[3]) == c["smin_sha256"]


def test_batch_matches_golden():
    keys = [(4, i) for i in range(8)]
    vols = [volume.workload(*k) for k in keys]
    B = Batch([(v.X, v.Y, v.Z) for v in vols])
    for i, v in enumerate(vols):
        B.set_tweights(i, v.capS, v.capT)
        for ax in range(3):
            B.set_nweights(i, ax, v.n[ax])
    flows = B.max_flow()
    for i, k in enumerate(keys):
        c = CASES[k]
        assert flows[i] == c["flow"]
        assert sha(B.fill_segments(i, mask=1, which=SOURCE)) == c["smin_sha256"]
        assert sha(B.fill_segments(i, mask=1, which=SINK)) == c["treach_sha256"]
    B.close()


def test_edge_cases():
    # all zero: nothing flows, nothing reachable
    X, Y, Z = 10, 9, 3
    N = X * Y * Z
    z = np.zeros(N, np.int32)
    flow, smin, treach, _ = solve(X, Y, Z, z, z, [z, z, z])
    assert flow == 0 and smin.sum() == 0 and treach.sum() == 0
    # t-links only: flow is the sum of min(capS, capT)
    rng = np.random.default_rng(0)
    s, t = rng.integers(0, 50, N).astype(np.int32), rng.integers(0, 50, N).astype(np.int32)
    flow, smin, treach, _ = solve(X, Y, Z, s, t, [z, z, z])
    assert flow == int(np.minimum(s, t).sum())
    assert np.array_equal(smin.astype(bool), s > t) and np.array_equal(treach.astype(bool), t > s)


def test_errors_are_loud():
    X, Y, Z = 8, 8, 8
    N = X * Y * Z
    g = GridGraph(X, Y, Z)
    with pytest.raises(_lib.CgcError) as e:
        g.fill_segments()
    assert e.value.code == 7  # CGC_ERR_STATE before max_flow
    with pytest.raises(_lib.CgcError) as e:
        g.max_flow()
    assert e.value.code == 7  # no t-links yet
    big = np.full(N, 2**31 - 1, np.int32)
    g.set_tweights(big, np.zeros(N, np.int32))
    for ax in range(3):
        g.set_nweights(ax, big)
    with pytest.raises(_lib.CgcError) as e:
        g.max_flow()
    assert e.value.code == 6  # CGC_ERR_OVERFLOW
    g.close()


def test_resolve_after_reupload_is_identical():
    X, Y, Z = 24, 16, 12
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 77)
    g = GridGraph(X, Y, Z)
    res = []
    for _ in range(3):
        g.set_tweights(capS, capT)
        for ax in range(3):
            g.set_nweights(ax, fwd[ax], bwd[ax])
        res.append((g.max_flow(), sha(g.fill_segments(which=SOURCE)), sha(g.fill_segments(which=SINK))))
    with pytest.raises(_lib.CgcError):
        g.max_flow()  # capacities were consumed by the last solve
    g.close()
    assert res[0] == res[1] == res[2]
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    assert res[0][0] == f0


def _face_case(X=16, Y=8, Z=8, sink_x=7, src_x=12, nlink=5):
    """Sink capacity only on the +x face of the first tile, source capacity only
    inside the second tile: the BFS seeds sit on a tile face and the second
    tile has none of its own."""
    N = X * Y * Z
    capS = np.zeros((Z, Y, X), np.int32)
    capT = np.zeros((Z, Y, X), np.int32)
    capT[:, :, sink_x] = 3
    capS[:, :, src_x] = 7
    fx = np.full((Z, Y, X), nlink, np.int32)
    fx[:, :, -1] = 0
    z = np.zeros(N, np.int32)
    return X, Y, Z, capS.reshape(-1), capT.reshape(-1), [fx.reshape(-1), z, z]


@pytest.mark.parametrize("policy", ["default", "host_loop", "cta3_L2_R4", "cta4_no_region", "excl"])
@pytest.mark.parametrize("sink_x,src_x", [(7, 12), (8, 3), (7, 8), (0, 15)])
def test_seeds_on_tile_faces(sink_x, src_x, policy):
    X, Y, Z, capS, capT, fwd = _face_case(sink_x=sink_x, src_x=src_x)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd)
    flow, smin, treach, _ = solve(X, Y, Z, capS, capT, fwd, None, POLICIES[policy])
    assert f0 > 0
    assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


@pytest.mark.parametrize("policy", ["default", "host_loop", "cta3_L2_R4", "cta4_no_region", "excl"])
@pytest.mark.parametrize("seed", range(8))
def test_sparse_terminals_match_oracle(seed, policy):
    """Very few t-links on a well connected grid: seeds land on tile faces and
    many tiles have none (exercises BFS and reachability across tiles)."""
    X, Y, Z = 40, 24, 17
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 500 + seed, zero_frac=0.995, nmax=30)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    flow, smin, treach, _ = solve(X, Y, Z, capS, capT, fwd, bwd, POLICIES[policy])
    assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


@pytest.mark.parametrize("policy", ["default", "host_loop", "no_region", "cta3_L2_R4", "cta4_no_region",
                                    "bfsw_all", "excl", "excl_cta3_L1_K1"])
@pytest.mark.parametrize("axis,n", [(0, 2), (0, 9), (0, 16), (0, 40), (1, 17), (2, 24), (0, 64)])
def test_chain_through_every_voxel(axis, n, policy):
    """A 1-D chain with the source at one end and the sink at the other: the
    first voxel's distance to the sink is the voxel count itself."""
    dims = [1, 1, 1]
    dims[axis] = n
    X, Y, Z = dims
    capS = np.zeros(n, np.int32)
    capT = np.zeros(n, np.int32)
    capS[0] = 50
    capT[-1] = 50
    chain = np.full(n, 9, np.int32)
    chain[(n - 1) // 2] = 3
    chain[-1] = 0
    z = np.zeros(n, np.int32)
    fwd = [z, z, z]
    fwd[axis] = chain
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd)
    flow, smin, treach, _ = solve(X, Y, Z, capS, capT, fwd, None, POLICIES[policy])
    assert f0 == 3
    assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


def test_snake_path_longer_than_a_tile():
    """One long winding path through a 2-D grid (every voxel on it): the
    distance to the sink is the voxel count, far beyond a tile."""
    X, Y = 24, 16
    N = X * Y
    order = [(x if y % 2 == 0 else X - 1 - x, y) for y in range(Y) for x in range(X)]
    fx = np.zeros((Y, X), np.int32)
    fy = np.zeros((Y, X), np.int32)
    for (x0, y0), (x1, y1) in zip(order, order[1:]):
        if y0 == y1:
            fx[y0, min(x0, x1)] = 7
        else:
            fy[min(y0, y1), x0] = 7
    capS = np.zeros((Y, X), np.int32)
    capT = np.zeros((Y, X), np.int32)
    capS[order[0][1], order[0][0]] = 100
    capT[order[-1][1], order[-1][0]] = 100
    z = np.zeros(N, np.int32)
    fwd = [fx.reshape(-1), fy.reshape(-1), z]
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, 1, capS.reshape(-1), capT.reshape(-1), fwd)
    assert f0 == 7
    for pol in (None, Policy(persistent=-1), Policy(region_relabels=-1, local_pulses=2), POLICIES["cta3_L2_R4"],
                POLICIES["cta4_no_region"], Policy(ctas_per_sm=4, region_relabels=-1, local_pulses=2),
                POLICIES["cta4_bfsw_K2"]):
        flow, smin, treach, _ = solve(X, Y, 1, capS.reshape(-1), capT.reshape(-1), fwd, None, pol)
        assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0)


def _random_scheduler_weights(seed):
    """Untrained (random) scheduler weights: the learned schedule must still be exact."""
    import ctypes as C
    lib = _lib.load()
    h = C.c_void_p()
    _lib.check(lib.cgc_trainer_create(1, 4, seed, C.byref(h)))
    conv = np.zeros(3 * 27 * 256, np.uint16)
    head = np.zeros(34, np.float32)
    _lib.check(lib.cgc_trainer_weights(h, conv.ctypes.data, head.ctypes.data))
    lib.cgc_trainer_destroy(h)
    head[32:] = [0.0, 3.0]  # make budgets large and priorities mixed
    _lib.check(lib.cgc_scheduler_load(conv.ctypes.data, head.ctypes.data))


@pytest.mark.parametrize("learned", [1, 2, 3])
@pytest.mark.parametrize("key", [(1, 0), (4, 1), (2, 0)])
def test_learned_scheduler_is_exact(key, learned):
    """Budgets and priorities only reorder pushes and relabels: flow and both
    cut sets stay bit-identical, with the committed weights and random ones."""
    from cugip_b200 import scheduler
    c = CASES[key]
    v = volume.workload(*key)
    for weights in ("committed", 7, 8):
        if weights == "committed":
            if not os.path.exists(scheduler.WEIGHTS):
                continue
            scheduler.load_weights()
        else:
            _random_scheduler_weights(weights)
        for pol in (Policy(learned=learned), Policy(learned=learned, ctas_per_sm=3, local_pulses=2, region_relabels=4,
                                                    sweeps_per_relabel=4),
                    Policy(learned=learned, ctas_per_sm=4, region_relabels=4, bfs_warp_min=8),
                    Policy(learned=learned, exclusive=1, ctas_per_sm=3)):
            flow, smin, treach, st = solve(v.X, v.Y, v.Z, v.capS, v.capT, v.n, None, pol)
            assert flow == c["flow"] and sha(smin) == c["smin_sha256"] and sha(treach) == c["treach_sha256"]


def test_scheduling_traces_are_recorded():
    from cugip_b200 import scheduler
    v = volume.workload(5, 3)
    g = GridGraph(v.X, v.Y, v.Z)
    g.set_tweights(v.capS, v.capT)
    for ax in range(3):
        g.set_nweights(ax, v.n[ax])
    g.max_flow(scheduler.TRACE_POLICY)
    feat, pulses, sink = g.sched_trace()
    g.close()
    assert feat.shape[0] >= 1 and feat.shape[1] == 16 ** 3
    import torch
    f = torch.from_numpy(feat.astype(np.int16)).view(torch.bfloat16).float().numpy()
    active = f[:, :, 1] > 0
    assert active.any()
    assert (pulses[active] > 0).all()          # every active tile was visited
    assert not (f[~active] != 0).any()         # inactive tiles have zero features


def _device_cut_capacity(capS, capT, fwd, bwd, side):
    """Capacity of the cut (side = source set) on the device, in int64, one z
    slice of the (Z, Y, X) volumes at a time: capT over the source side, capS
    over the rest, n-links from the source side to the rest."""
    import torch
    Z = side.shape[0]
    total = 0
    for z in range(Z):
        s = side[z].bool()
        total += int(capT[z][s].sum(dtype=torch.int64)) + int(capS[z][~s].sum(dtype=torch.int64))
        # x and y links inside the slice: v -> v+e with fwd[v], v+e -> v with bwd[v]
        for ax, (f, b) in enumerate(((fwd[0][z], bwd[0][z]), (fwd[1][z], bwd[1][z]))):
            if ax == 0:
                a, c, fa, ba = s[:, :-1], s[:, 1:], f[:, :-1], b[:, :-1]
            else:
                a, c, fa, ba = s[:-1, :], s[1:, :], f[:-1, :], b[:-1, :]
            total += int(fa[a & ~c].sum(dtype=torch.int64)) + int(ba[~a & c].sum(dtype=torch.int64))
        if z + 1 < Z:
            c = side[z + 1].bool()
            total += int(fwd[2][z][s & ~c].sum(dtype=torch.int64)) + int(bwd[2][z][~s & c].sum(dtype=torch.int64))
    return total


def test_largest_grid_certificate():
    """768^3 (453 M voxels; the residual planes span more than 2^31 entries):
    random capacities made on the device, solved through the device API; both
    returned cuts -- the minimal source side and the complement of the sink
    side -- have a capacity equal to the flow, which certifies a maximum flow
    and a minimum cut without a CPU solve."""
    import torch
    dev = torch.device("cuda", 0)
    n = 768
    if torch.cuda.get_device_properties(0).total_memory < 80 * 2 ** 30:
        pytest.skip("needs a GPU with 80 GB or more")
    g = torch.Generator(device=dev)
    g.manual_seed(768)

    def plane(hi, zero_frac):
        p = torch.randint(0, hi, (n, n, n), generator=g, device=dev, dtype=torch.int32)
        p[torch.rand((n, n, n), generator=g, device=dev) < zero_frac] = 0
        return p

    capS, capT = plane(60, 0.7), plane(60, 0.7)
    fwd = [plane(40, 0.2) for _ in range(3)]
    # no capacity leaves the grid
    fwd[0][:, :, -1] = 0
    fwd[1][:, -1, :] = 0
    fwd[2][-1, :, :] = 0
    G = GridGraph(n, n, n)
    try:
        G.set_tweights_device(capS.data_ptr(), capT.data_ptr())
        for ax in range(3):
            G.set_nweights_device(ax, fwd[ax].data_ptr())
        flow = G.max_flow()
        smin = torch.empty((n, n, n), dtype=torch.uint8, device=dev)
        treach = torch.empty((n, n, n), dtype=torch.uint8, device=dev)
        G.fill_segments_device(smin.data_ptr(), 1, 0, SOURCE)
        G.fill_segments_device(treach.data_ptr(), 1, 0, SINK)
    finally:
        G.close()
    assert flow > 0
    assert not bool((smin.bool() & treach.bool()).any())  # a source-side voxel cannot reach the sink
    assert _device_cut_capacity(capS, capT, fwd, fwd, smin) == flow
    assert _device_cut_capacity(capS, capT, fwd, fwd, 1 - treach) == flow


def test_host_setters_copy_before_returning():
    """The setters' contract (the reference copies at call time): once a setter
    returns, the caller may overwrite its arrays -- here pinned ones, whose
    copies would otherwise still be in flight."""
    import torch
    X, Y, Z = 48, 40, 24
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, 4242)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (capS, capT, *fwd, *bwd)]
    host = [t.numpy() for t in pin]
    g = GridGraph(X, Y, Z)
    try:
        for rep in range(2):
            for t, a in zip(pin, (capS, capT, *fwd, *bwd)):
                t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
            g.set_tweights(host[0], host[1])
            host[0][:] = 7777
            host[1][:] = 0
            for ax in range(3):
                g.set_nweights(ax, host[2 + ax], host[5 + ax])
                host[2 + ax][:] = 12345
                host[5 + ax][:] = 0
            assert g.max_flow() == f0
            assert np.array_equal(g.fill_segments(mask=1, which=SOURCE), s0)
            assert np.array_equal(g.fill_segments(mask=1, which=SINK), t0)
    finally:
        g.close()
