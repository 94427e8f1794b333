"""Graph builders shared by the tests: the reference's own test graphs and
seeded random grids."""
from __future__ import annotations

import numpy as np


def four_by_four():
    """test/graph_cut.cu:13-67 of the reference: a 4x4 grid, horizontal caps 5,
    vertical caps 5 except rows 1->2 (cap 1), source caps 100 on row 0, sink caps
    100 on row 3.  Max flow 4."""
    v1 = [0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11]
    v2 = [1, 2, 3, 5, 6, 7, 9, 10, 11, 13, 14, 15, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15]
    w = [5] * 12 + [5, 5, 5, 5, 1, 1, 1, 1, 5, 5, 5, 5]
    capS = [100] * 4 + [0] * 12
    capT = [0] * 12 + [100] * 4
    return 16, np.array(v1), np.array(v2), np.array(w), np.array(w), np.array(capS), np.array(capT)


def layered(layers=100, size=1024, nbrs=8, flip=False):
    """unit_tests/graph_cut_test.cu:22-67 of the reference: `layers` layers of
    `size` vertices, vertex i of layer L-1 joined to vertices (i+j)%size of layer
    L (j < nbrs); forward cap 1 in the middle layer and 20 elsewhere, backward
    cap twice the forward cap; source cap 100000 on the first layer, sink on the
    last (swapped with flip).  Max flow 8192 (flip: 16384) for 100x1024x8."""
    a, b, f, g = [], [], [], []
    for L in range(1, layers):
        w = 1 if L == layers // 2 else 20
        i = np.arange(size)
        for j in range(nbrs):
            a.append((L - 1) * size + i)
            b.append(L * size + (i + j) % size)
            f.append(np.full(size, w))
            g.append(np.full(size, 2 * w))
    a, b, f, g = (np.concatenate(x) for x in (a, b, f, g))
    n = layers * size
    src = np.zeros(n, np.int64)
    snk = np.zeros(n, np.int64)
    src[:size] = 100000
    snk[-size:] = 100000
    if flip:
        src, snk = snk, src
    return n, a, b, f, g, src, snk


def random_grid(X, Y, Z, seed, tmax=60, nmax=40, asym=True, zero_frac=0.2):
    """Seeded random grid: t-links and (optionally asymmetric) n-links, some zeros."""
    rng = np.random.default_rng(seed)
    N = X * Y * Z
    capS = rng.integers(0, tmax, N).astype(np.int32)
    capT = rng.integers(0, tmax, N).astype(np.int32)
    capS[rng.random(N) < zero_frac] = 0
    capT[rng.random(N) < zero_frac] = 0
    fwd, bwd = [], []
    shape = (Z, Y, X)
    for ax_np in (2, 1, 0):
        f = rng.integers(0, nmax, N).astype(np.int32).reshape(shape)
        b = rng.integers(0, nmax, N).astype(np.int32).reshape(shape) if asym else f.copy()
        idx = [slice(None)] * 3
        idx[ax_np] = -1
        f[tuple(idx)] = 0
        b[tuple(idx)] = 0
        fwd.append(f.reshape(-1))
        bwd.append(b.reshape(-1))
    return capS, capT, fwd, bwd


def grid_edges(X, Y, Z, fwd, bwd):
    """Edge list (a, b, cap a->b, cap b->a) of a grid in linear ids."""
    ids = np.arange(X * Y * Z).reshape(Z, Y, X)
    A, B, F, G = [], [], [], []
    for ax, ax_np in ((0, 2), (1, 1), (2, 0)):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax_np] = slice(0, -1)
        hi[ax_np] = slice(1, None)
        A.append(ids[tuple(lo)].reshape(-1))
        B.append(ids[tuple(hi)].reshape(-1))
        F.append(np.asarray(fwd[ax]).reshape(Z, Y, X)[tuple(lo)].reshape(-1))
        G.append(np.asarray(bwd[ax]).reshape(Z, Y, X)[tuple(lo)].reshape(-1))
    return (np.concatenate(A), np.concatenate(B), np.concatenate(F), np.concatenate(G))
