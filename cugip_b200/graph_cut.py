"""Host-side mirror of cugip's graph-cut interface over the C ABI of libcgc.

`Graph` keeps the names, argument meaning and error behaviour of
`cugip::Graph<TFlow>` (include/cugip/advanced_operations/graph_cut.hpp:47-146):
set_vertex_count / set_nweights(edge list) / set_tweights / max_flow /
fill_segments, with int32 capacities and an exact int flow.  `GridGraph` is
the grid-native form: t-link volumes and one n-link volume per axis, which is
what the reference's grid front-end builds
(benchmarks/graph_cut/graph_cut.cpp:33-98).  `GenericGraph` takes any edge
list (the generic engine `Graph` falls back to when the edges do not form a
grid).  `Batch` solves many grids of uneven sizes in one launch.

Every solve runs on the GPU through libcgc.so; nothing here computes a flow.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import CgcError, check

SINK = "sink"      # vertices that can reach the sink (reference fill_segments semantics)
SOURCE = "source"  # vertices reachable from the source (minimal source side: the canonical cut)


def _which(which: str) -> int:
    if which in (SINK, _lib.SEG_SINK_REACH):
        return _lib.SEG_SINK_REACH
    if which in (SOURCE, _lib.SEG_SOURCE_MIN):
        return _lib.SEG_SOURCE_MIN
    raise ValueError(f"unknown segment set {which!r}")


def _i32(a, n: int, name: str) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a).reshape(-1))
    if arr.dtype != np.int32:
        if arr.dtype.kind == "f":
            if not np.all(np.isfinite(arr)) or not np.all(arr == np.round(arr)):
                raise CgcError(1, f"{name}: capacities must be integral (the engine is exact)")
        if arr.size and (arr.min() < 0 or arr.max() > np.iinfo(np.int32).max):
            raise CgcError(1, f"{name}: capacities must be in [0, 2^31)")
        arr = arr.astype(np.int32)
    if arr.size != n:
        raise CgcError(1, f"{name}: expected {n} entries, got {arr.size}")
    return arr


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Policy:
    """Runtime counterpart of GraphCutPolicy (detail/graph_cut_policies.hpp:23-89).

    Every field is a cgc_options field (include/cgc.h); 0 means the default."""

    def __init__(self, local_pulses: int = 0, sweeps_per_relabel: int = 0, wait_limit_us: int = 0,
                 max_sweeps: int = 0, persistent: int = 0, region_relabels: int = 0, stall_sweeps: int = 0,
                 ctas_per_sm: int = 0, learned: int = 0, trace_cycles: int = 0, bfs_warp_min: int = 0,
                 exclusive: int = 0, relabel: int = 0):
        self.local_pulses = local_pulses
        self.sweeps_per_relabel = sweeps_per_relabel
        self.wait_limit_us = wait_limit_us
        self.max_sweeps = max_sweeps
        self.persistent = persistent
        self.region_relabels = region_relabels
        self.stall_sweeps = stall_sweeps
        self.ctas_per_sm = ctas_per_sm
        self.learned = learned
        self.trace_cycles = trace_cycles
        self.bfs_warp_min = bfs_warp_min
        self.exclusive = exclusive
        self.relabel = relabel

    def options(self) -> _lib.Options:
        return _lib.options(**{k: getattr(self, k) for k in _lib.OPTION_FIELDS})

    @classmethod
    def from_options(cls, o: _lib.Options) -> "Policy":
        return cls(**{k: getattr(o, k) for k in _lib.OPTION_FIELDS})

    def __repr__(self):
        return (f"Policy(L={self.local_pulses}, R={self.region_relabels}, K={self.sweeps_per_relabel}, "
                f"ctas={self.ctas_per_sm}, stall={self.stall_sweeps}, learned={self.learned}, "
                f"bfsw={self.bfs_warp_min}, excl={self.exclusive}, relabel={self.relabel})")

    def with_(self, **kw) -> "Policy":
        p = Policy.from_options(self.options())
        for k, v in kw.items():
            setattr(p, k, v)
        return p


def _autotune(fn, handle, candidates, repeats):
    best = _lib.Options()
    ms = C.c_double()
    if candidates:
        arr = (_lib.Options * len(candidates))(*[c.options() for c in candidates])
        check(fn(handle, arr, len(candidates), repeats, C.byref(best), C.byref(ms)))
    else:
        check(fn(handle, None, 0, repeats, C.byref(best), C.byref(ms)))
    return Policy.from_options(best), float(ms.value)


def autotune_lookup(voxels: int, instances: int = 1) -> Policy | None:
    o = _lib.Options()
    rc = _lib.load().cgc_autotune_lookup(int(voxels), int(instances), C.byref(o))
    return Policy.from_options(o) if rc == 0 else None


class GridGraph:
    """X*Y*Z 6-connected grid graph; vertex id = x + X*(y + Y*z)."""

    def __init__(self, X: int, Y: int, Z: int = 1, stream: int | None = None):
        self._lib = _lib.load()
        self.X, self.Y, self.Z = int(X), int(Y), int(Z)
        self.n = self.X * self.Y * self.Z
        h = C.c_void_p()
        check(self._lib.cgc_grid_create(self.X, self.Y, self.Z, C.c_void_p(stream or 0), C.byref(h)))
        self._h = h
        self.flow: int | None = None

    @classmethod
    def _wrap(cls, handle: C.c_void_p, dims) -> "GridGraph":
        g = cls.__new__(cls)
        g._lib = _lib.load()
        g.X, g.Y, g.Z = (int(d) for d in dims)
        g.n = g.X * g.Y * g.Z
        g._h = handle
        g.flow = None
        return g

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cgc_grid_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- capacities ---------------------------------------------------------
    def set_tweights(self, cap_source, cap_sink) -> None:
        s = _i32(cap_source, self.n, "cap_source")
        t = _i32(cap_sink, self.n, "cap_sink")
        check(self._lib.cgc_grid_set_tlinks(self._h, _ptr(s), _ptr(t)))

    def set_nweights(self, axis: int, forward, backward=None) -> None:
        """n-links along `axis` (0=x,1=y,2=z): forward[v] = cap v -> v+e_axis,
        backward[v] = cap v+e_axis -> v (same as forward when omitted)."""
        f = _i32(forward, self.n, "forward")
        b = f if backward is None else _i32(backward, self.n, "backward")
        check(self._lib.cgc_grid_set_nlinks(self._h, int(axis), _ptr(f), _ptr(b)))

    def set_tweights_device(self, cap_source_ptr: int, cap_sink_ptr: int) -> None:
        check(self._lib.cgc_grid_set_tlinks_device(self._h, C.c_void_p(cap_source_ptr), C.c_void_p(cap_sink_ptr)))

    def set_nweights_device(self, axis: int, forward_ptr: int, backward_ptr: int | None = None) -> None:
        b = forward_ptr if backward_ptr is None else backward_ptr
        check(self._lib.cgc_grid_set_nlinks_device(self._h, int(axis), C.c_void_p(forward_ptr), C.c_void_p(b)))

    # -- solve --------------------------------------------------------------
    def max_flow(self, policy: Policy | None = None) -> int:
        flow = C.c_int64()
        opts = policy.options() if policy else None
        check(self._lib.cgc_grid_maxflow(self._h, C.byref(opts) if opts else None, C.byref(flow)))
        self.flow = int(flow.value)
        return self.flow

    def max_flow_async(self, policy: Policy | None = None) -> None:
        """Queues the solve of the capacities set so far on the grid's stream and
        returns at once; wait() blocks until it is done and returns the flow.
        Meanwhile another grid's set_* calls can copy its inputs to the device,
        so uploads and solves of consecutive grids overlap."""
        opts = policy.options() if policy else None
        check(self._lib.cgc_grid_maxflow_async(self._h, C.byref(opts) if opts else None))

    def wait(self) -> int:
        flow = C.c_int64()
        check(self._lib.cgc_grid_wait(self._h, C.byref(flow)))
        self.flow = int(flow.value)
        return self.flow

    def fill_segments(self, out: np.ndarray | None = None, mask: int = 255, background: int = 0,
                      which: str = SINK) -> np.ndarray:
        """out[v] = mask where v is in the chosen set, else background.
        which=SINK: vertices that can reach the sink (cugip's fill_segments,
        graph_cut.hpp:304-333); which=SOURCE: vertices reachable from the source
        (the canonical minimum cut)."""
        if out is None:
            out = np.empty(self.n, dtype=np.uint8)
        if out.dtype != np.uint8 or not out.flags["C_CONTIGUOUS"] or out.size != self.n:
            raise CgcError(1, "fill_segments: out must be a contiguous uint8 array of n entries")
        check(self._lib.cgc_grid_get_segments(self._h, _which(which), _ptr(out), mask, background))
        return out

    def fill_segments_device(self, out_ptr: int, mask: int = 255, background: int = 0, which: str = SINK) -> None:
        check(self._lib.cgc_grid_get_segments_device(self._h, _which(which), C.c_void_p(out_ptr), mask, background))

    def residuals(self) -> dict:
        """Final residual capacities in linear layout: r (6,n) for +x,-x,+y,-y,+z,-z, resT and excess."""
        r = np.empty((6, self.n), dtype=np.int32)
        rt = np.empty(self.n, dtype=np.int32)
        ex = np.empty(self.n, dtype=np.int32)
        ptrs = (C.c_void_p * 6)(*[r[d].ctypes.data for d in range(6)])
        check(self._lib.cgc_grid_get_residuals(self._h, ptrs, _ptr(rt), _ptr(ex)))
        return {"r": r, "resT": rt, "excess": ex}

    def labels(self) -> np.ndarray:
        """Distance to the sink after the final global relabel, per voxel (linear
        layout); INT32_MIN where the sink cannot be reached."""
        out = np.empty(self.n, dtype=np.int32)
        check(self._lib.cgc_grid_get_labels(self._h, _ptr(out)))
        return out

    def stats(self) -> dict:
        s = _lib.Stats()
        check(self._lib.cgc_grid_stats(self._h, C.byref(s)))
        return s.as_dict()

    def trace(self) -> list:
        return _read_trace(self._lib.cgc_grid_trace, self._h)

    def sched_trace(self, max_cycles: int = 64):
        """Scheduling traces of the last solve (Policy.trace_cycles > 0): features
        (cycles, T, 16) as uint16 BF16 bits, first-visit pulses (cycles, T) and
        sink delivery (cycles, T)."""
        n = C.c_int32()
        check(self._lib.cgc_grid_sched_trace(self._h, None, None, None, 0, C.byref(n)))
        c = min(n.value, max_cycles)
        T = ((self.X + 7) // 8) * ((self.Y + 7) // 8) * ((self.Z + 7) // 8)
        feat = np.zeros((c, T, 16), np.uint16)
        pulses = np.zeros((c, T), np.uint8)
        sink = np.zeros((c, T), np.uint8)
        if c:
            check(self._lib.cgc_grid_sched_trace(self._h, feat.ctypes.data, pulses.ctypes.data, sink.ctypes.data, c,
                                                 C.byref(n)))
        return feat, pulses, sink

    def autotune(self, candidates: list | None = None, repeats: int = 1):
        """Fastest policy for the current capacities (which stay set): (policy, ms)."""
        return _autotune(self._lib.cgc_grid_autotune, self._h, candidates, repeats)


TRACE_KINDS = {1: "bfs_round", 2: "relabel_done", 3: "sweep", 4: "reach_round", 5: "flow"}


def _read_trace(fn, handle) -> list:
    n = C.c_int32()
    check(fn(handle, None, 0, C.byref(n)))
    buf = np.zeros(2 * max(n.value, 1), dtype=np.int64)
    check(fn(handle, buf.ctypes.data_as(C.c_void_p), n.value, C.byref(n)))
    out = []
    for i in range(n.value):
        w = int(buf[2 * i]) & 0xFFFFFFFFFFFFFFFF
        rec = {"kind": TRACE_KINDS.get(w >> 56, w >> 56), "index": (w >> 24) & 0xFFFFFFFF, "tiles": w & 0xFFFFFF}
        rec["flow" if (w >> 56) == 5 else "ns"] = int(buf[2 * i + 1])
        out.append(rec)
    return out


class GenericGraph:
    """Any edge list solved on the GPU (the non-grid path of cugip::Graph):
    n vertices, edge i joins a[i] and b[i] with capacity cap_ab[i] from a[i]
    to b[i] and cap_ba[i] back (cgc_graph_* in cgc.h)."""

    def __init__(self, n: int, a, b, cap_ab, cap_ba, stream: int | None = None):
        self._lib = _lib.load()
        self.n = int(n)
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int64).reshape(-1))
        b = np.ascontiguousarray(np.asarray(b, dtype=np.int64).reshape(-1))
        if a.size != b.size:
            raise CgcError(1, "a and b must have the same length")
        m = a.size
        if m and (min(a.min(), b.min()) < 0 or max(a.max(), b.max()) >= self.n):
            raise CgcError(1, "edge endpoints must lie in [0, n)")
        a32, b32 = a.astype(np.int32), b.astype(np.int32)
        f = _i32(cap_ab, m, "cap_ab")
        w = _i32(cap_ba, m, "cap_ba")
        h = C.c_void_p()
        check(self._lib.cgc_graph_create(self.n, m, _ptr(a32), _ptr(b32), _ptr(f), _ptr(w), C.c_void_p(stream or 0),
                                         C.byref(h)))
        self._h = h
        self.flow: int | None = None

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cgc_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_tweights(self, cap_source, cap_sink) -> None:
        check(self._lib.cgc_graph_set_tlinks(self._h, _ptr(_i32(cap_source, self.n, "cap_source")),
                                             _ptr(_i32(cap_sink, self.n, "cap_sink"))))

    def max_flow(self, policy: Policy | None = None) -> int:
        f = C.c_int64()
        opts = policy.options() if policy is not None else None
        check(self._lib.cgc_graph_maxflow(self._h, C.byref(opts) if opts is not None else None, C.byref(f)))
        self.flow = int(f.value)
        return self.flow

    def fill_segments(self, out=None, mask: int = 255, background: int = 0, which: str = SINK):
        seg = np.empty(self.n, np.uint8)
        check(self._lib.cgc_graph_get_segments(self._h, _which(which), _ptr(seg), mask, background))
        if out is None:
            return seg
        out[...] = seg.reshape(np.shape(out))
        return out

    def stats(self) -> dict:
        s = _lib.Stats()
        check(self._lib.cgc_graph_stats(self._h, C.byref(s)))
        return s.as_dict()


class Graph:
    """Mirror of cugip::Graph<TFlow> (graph_cut.hpp:47-146) for int32 capacities.

    Edges are EdgeRecord(first, second) pairs with forward = cap first->second
    and backward = cap second->first.  An edge list that forms a 6-connected
    grid with linear vertex ids (see cgc_grid_create_from_edges) goes to the
    tile engine; any other graph goes to the generic CSR engine.
    """

    def __init__(self):
        self._n = 0
        self._solver: GridGraph | GenericGraph | None = None
        self._pending_t = None

    def set_vertex_count(self, count: int) -> None:
        self._n = int(count)
        self._solver = None

    def set_nweights(self, edge_count: int, edges, weights_forward, weights_backward) -> None:
        e = np.ascontiguousarray(np.asarray(edges, dtype=np.int64).reshape(-1, 2)[:edge_count])
        a = np.ascontiguousarray(e[:, 0].astype(np.uint32))
        b = np.ascontiguousarray(e[:, 1].astype(np.uint32))
        f = _i32(np.asarray(weights_forward)[:edge_count], edge_count, "weights_forward")
        w = _i32(np.asarray(weights_backward)[:edge_count], edge_count, "weights_backward")
        h = C.c_void_p()
        dims = (C.c_int32 * 3)()
        lib = _lib.load()
        rc = lib.cgc_grid_create_from_edges(self._n, edge_count, _ptr(a), _ptr(b), _ptr(f), _ptr(w),
                                            None, C.byref(h), dims)
        if rc == 8:  # CGC_ERR_NOT_GRID: the generic engine takes it
            self._solver = GenericGraph(self._n, e[:, 0], e[:, 1], f, w)
        else:
            check(rc)
            self._solver = GridGraph._wrap(h, list(dims))
        if self._pending_t is not None:
            self._solver.set_tweights(*self._pending_t)

    def set_tweights(self, cap_source, cap_sink) -> None:
        # the reference accepts t-links before n-links; keep them for the graph
        # set_nweights builds next
        self._pending_t = (_i32(cap_source, self._n, "cap_source"), _i32(cap_sink, self._n, "cap_sink"))
        if self._solver is not None:
            self._solver.set_tweights(*self._pending_t)

    def max_flow(self, policy: Policy | None = None) -> int:
        if self._solver is None:
            raise CgcError(7, "max_flow: set_nweights was not called")
        return self._solver.max_flow(policy)

    def fill_segments(self, out=None, mask: int = 255, background: int = 0, which: str = SINK):
        if self._solver is None:
            raise CgcError(7, "fill_segments: no graph")
        seg = self._solver.fill_segments(None, mask, background, which)
        if out is None:
            return seg
        out[...] = seg.reshape(np.shape(out))
        return out

    def stats(self) -> dict:
        if self._solver is None:
            raise CgcError(7, "stats: no graph")
        return self._solver.stats()

    @property
    def grid(self) -> GridGraph | None:
        return self._solver if isinstance(self._solver, GridGraph) else None

    @property
    def generic(self) -> GenericGraph | None:
        return self._solver if isinstance(self._solver, GenericGraph) else None


class Batch:
    """Many grid instances of uneven sizes solved by one launch."""

    def __init__(self, extents: Sequence[Sequence[int]], stream: int | None = None):
        self._lib = _lib.load()
        ext = np.ascontiguousarray(np.asarray(extents, dtype=np.int32).reshape(-1, 3))
        self.extents = [tuple(int(v) for v in row) for row in ext]
        h = C.c_void_p()
        check(self._lib.cgc_batch_create(len(self.extents), _ptr(ext), C.c_void_p(stream or 0), C.byref(h)))
        self._h = h
        self.flows: list[int] | None = None

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cgc_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _n(self, i: int) -> int:
        X, Y, Z = self.extents[i]
        return X * Y * Z

    def set_tweights(self, i: int, cap_source, cap_sink) -> None:
        n = self._n(i)
        check(self._lib.cgc_batch_set_tlinks(self._h, i, _ptr(_i32(cap_source, n, "cap_source")),
                                             _ptr(_i32(cap_sink, n, "cap_sink"))))

    def set_nweights(self, i: int, axis: int, forward, backward=None) -> None:
        n = self._n(i)
        f = _i32(forward, n, "forward")
        b = f if backward is None else _i32(backward, n, "backward")
        check(self._lib.cgc_batch_set_nlinks(self._h, i, int(axis), _ptr(f), _ptr(b)))

    def max_flow(self, policy: Policy | None = None) -> list[int]:
        flows = np.zeros(len(self.extents), dtype=np.int64)
        opts = policy.options() if policy else None
        check(self._lib.cgc_batch_maxflow(self._h, C.byref(opts) if opts else None,
                                          flows.ctypes.data_as(_lib.P64)))
        self.flows = [int(f) for f in flows]
        return self.flows

    def fill_segments(self, i: int, mask: int = 255, background: int = 0, which: str = SINK) -> np.ndarray:
        out = np.empty(self._n(i), dtype=np.uint8)
        check(self._lib.cgc_batch_get_segments(self._h, i, _which(which), _ptr(out), mask, background))
        return out

    def stats(self) -> dict:
        s = _lib.Stats()
        check(self._lib.cgc_batch_stats(self._h, C.byref(s)))
        return s.as_dict()

    def trace(self) -> list:
        return _read_trace(self._lib.cgc_batch_trace, self._h)

    # -- device-resident path (pointers to device memory, e.g. tensor.data_ptr())
    def bind_inputs(self, i: int, cap_source_ptr: int, cap_sink_ptr: int, forward_ptrs, backward_ptrs=None) -> None:
        f = (C.c_void_p * 3)(*[p or None for p in forward_ptrs])
        b = None if backward_ptrs is None else (C.c_void_p * 3)(*[p or None for p in backward_ptrs])
        check(self._lib.cgc_batch_bind_inputs(self._h, i, C.c_void_p(cap_source_ptr), C.c_void_p(cap_sink_ptr), f, b))

    def bind_outputs(self, i: int, source_side_ptr: int | None, sink_side_ptr: int | None) -> None:
        check(self._lib.cgc_batch_bind_outputs(self._h, i, C.c_void_p(source_side_ptr or 0),
                                               C.c_void_p(sink_side_ptr or 0)))

    def enqueue(self, policy: Policy | None = None, flows_ptr: int | None = None) -> None:
        opts = policy.options() if policy else None
        check(self._lib.cgc_batch_enqueue(self._h, C.byref(opts) if opts else None, C.c_void_p(flows_ptr or 0)))

    def graph_create(self, policy: Policy | None = None, flows_ptr: int | None = None) -> None:
        opts = policy.options() if policy else None
        check(self._lib.cgc_batch_graph_create(self._h, C.byref(opts) if opts else None, C.c_void_p(flows_ptr or 0)))

    def graph_launch(self) -> None:
        check(self._lib.cgc_batch_graph_launch(self._h))

    def autotune(self, candidates: list | None = None, repeats: int = 1):
        """Fastest policy for the current capacities or bound inputs: (policy, ms)."""
        return _autotune(self._lib.cgc_batch_autotune, self._h, candidates, repeats)

    def wait(self) -> list[int]:
        flows = np.zeros(len(self.extents), dtype=np.int64)
        check(self._lib.cgc_batch_wait(self._h, flows.ctypes.data_as(_lib.P64)))
        self.flows = [int(f) for f in flows]
        return self.flows
