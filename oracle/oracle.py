"""CPU oracle for the grid graph-cut path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg (and its
`--impl reference` arm) may import this module; the product path never does.

Wraps oracle/maxflow_oracle.c: a Boykov-Kolmogorov max-flow written from the
TPAMI 2004 paper (restating the reference's CPU path,
benchmarks/graph_cut/boykov_kolmogorov.cpp:20-83, whose BK301 library is not
vendored) and an independent Dinic solver.  Results: exact int64 flow, the
sink-reachable set (reference fill_segments / what_segment()==SINK semantics)
and the source-reachable set (canonical minimum cut).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
BK, DINIC = 0, 1

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "maxflow_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(src) > os.path.getmtime(LIB):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "liboracle.so"], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(LIB)
        vp = C.c_void_p
        lib.orc_maxflow_grid.restype = C.c_int
        lib.orc_maxflow_grid.argtypes = [C.c_int, C.c_int32, C.c_int32, C.c_int32] + [vp] * 8 + [vp, vp, vp, vp]
        lib.orc_maxflow_edges.restype = C.c_int
        lib.orc_maxflow_edges.argtypes = [C.c_int, C.c_int32, C.c_int64] + [vp] * 6 + [vp, vp, vp, vp]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _c32(a):
    return np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=np.int32)


def maxflow_grid(X, Y, Z, capS, capT, fwd, bwd=None, algo=BK):
    """fwd/bwd: 3 arrays (x,y,z) of N entries, fwd[a][v] = cap v -> v+e_a,
    bwd[a][v] = cap v+e_a -> v (symmetric when bwd is None).
    Returns (flow, smin uint8[N], treach uint8[N], seconds)."""
    lib = load()
    N = X * Y * Z
    capS, capT = _c32(capS), _c32(capT)
    f = [_c32(a) for a in fwd]
    b = f if bwd is None else [_c32(a) for a in bwd]
    flow = C.c_int64()
    secs = C.c_double()
    smin = np.empty(N, np.uint8)
    treach = np.empty(N, np.uint8)
    rc = lib.orc_maxflow_grid(algo, X, Y, Z, _p(capS), _p(capT), _p(f[0]), _p(b[0]), _p(f[1]), _p(b[1]),
                              _p(f[2]), _p(b[2]), C.byref(flow), _p(smin), _p(treach), C.byref(secs))
    if rc:
        raise RuntimeError(f"oracle failed ({rc})")
    return int(flow.value), smin, treach, float(secs.value)


def maxflow_edges(n, a, b, cab, cba, capS, capT, algo=BK):
    """Generic graph: edge i joins a[i], b[i] with caps cab (a->b) and cba (b->a)."""
    lib = load()
    a, b, cab, cba = _c32(a), _c32(b), _c32(cab), _c32(cba)
    capS, capT = _c32(capS), _c32(capT)
    flow = C.c_int64()
    secs = C.c_double()
    smin = np.empty(n, np.uint8)
    treach = np.empty(n, np.uint8)
    rc = lib.orc_maxflow_edges(algo, n, a.size, _p(a), _p(b), _p(cab), _p(cba), _p(capS), _p(capT),
                               C.byref(flow), _p(smin), _p(treach), C.byref(secs))
    if rc:
        raise RuntimeError(f"oracle failed ({rc})")
    return int(flow.value), smin, treach, float(secs.value)


def cut_capacity_grid(X, Y, Z, capS, capT, fwd, bwd, source_side):
    """Capacity of the cut (S = source_side, T = rest): sum of capT over S,
    capS over T and n-link capacities from S to T (int64)."""
    S = np.asarray(source_side).reshape(Z, Y, X).astype(bool)
    cs = _c32(capS).reshape(Z, Y, X).astype(np.int64)
    ct = _c32(capT).reshape(Z, Y, X).astype(np.int64)
    total = int(ct[S].sum() + cs[~S].sum())
    bwd = fwd if bwd is None else bwd
    for ax, axis_np in ((0, 2), (1, 1), (2, 0)):
        f = _c32(fwd[ax]).reshape(Z, Y, X).astype(np.int64)
        bb = _c32(bwd[ax]).reshape(Z, Y, X).astype(np.int64)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis_np] = slice(0, -1)
        hi[axis_np] = slice(1, None)
        Slo, Shi = S[tuple(lo)], S[tuple(hi)]
        total += int(f[tuple(lo)][Slo & ~Shi].sum())   # lo in S, hi in T: lo -> hi
        total += int(bb[tuple(lo)][~Slo & Shi].sum())  # hi in S, lo in T: hi -> lo
    return total
