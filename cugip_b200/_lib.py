"""ctypes binding of libcgc.so (the C ABI declared in include/cgc.h).

The library is the only compute path: if it is missing or cannot be loaded,
every call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# CGC_LIBRARY may name another build of the same ABI (the bounds-checked
# libcgc_bounds.so for test runs)
LIB_PATH = os.environ.get("CGC_LIBRARY") or os.path.join(HERE, "libcgc.so")

CGC_OK = 0
ERRORS = {
    1: "CGC_ERR_ARG", 2: "CGC_ERR_OOM", 3: "CGC_ERR_CUDA", 4: "CGC_ERR_TIMEOUT",
    5: "CGC_ERR_NOT_CONVERGED", 6: "CGC_ERR_OVERFLOW", 7: "CGC_ERR_STATE",
    8: "CGC_ERR_NOT_GRID", 9: "CGC_ERR_NO_DEVICE",
}
SEG_SINK_REACH = 0
SEG_SOURCE_MIN = 1


class CgcError(RuntimeError):
    """Raised for a non-zero status of a cgc_* call (mirrors the reference's
    ExceptionBase thrown by CUGIP_CHECK_RESULT, include/cugip/exception.hpp:33-47)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("struct_size", C.c_int32), ("local_pulses", C.c_int32), ("sweeps_per_relabel", C.c_int32),
                ("wait_limit_us", C.c_int32), ("max_sweeps", C.c_int32), ("persistent", C.c_int32),
                ("region_relabels", C.c_int32), ("stall_sweeps", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("learned", C.c_int32), ("trace_cycles", C.c_int32),
                ("bfs_warp_min", C.c_int32), ("exclusive", C.c_int32), ("relabel", C.c_int32),
                ("reserved", C.c_int32 * 2)]


class Stats(C.Structure):
    _fields_ = [("flow", C.c_int64), ("sweeps", C.c_int64), ("global_relabels", C.c_int64),
                ("bfs_rounds", C.c_int64), ("tiles_swept", C.c_int64), ("tiles_relabelled", C.c_int64),
                ("pulses", C.c_int64), ("solve_ms", C.c_double), ("kernel_ms", C.c_double),
                ("launches", C.c_int64), ("bfs_ms", C.c_double), ("sweep_ms", C.c_double),
                ("reach_ms", C.c_double), ("sched_ms", C.c_double), ("tiles_checked", C.c_int64),
                ("reserved", C.c_int64 * 1)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


P32 = C.POINTER(C.c_int32)
PU32 = C.POINTER(C.c_uint32)
PU8 = C.POINTER(C.c_uint8)
P64 = C.POINTER(C.c_int64)
VP = C.c_void_p

# name -> (restype, argtypes); every exported symbol of include/cgc.h
SIGNATURES = {
    "cgc_last_error": (C.c_char_p, []),
    "cgc_version": (C.c_char_p, []),
    "cgc_init": (C.c_int, [C.c_int]),
    "cgc_launch_count": (C.c_int64, []),
    "cgc_grid_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, VP, C.POINTER(VP)]),
    "cgc_grid_destroy": (C.c_int, [VP]),
    "cgc_grid_set_tlinks": (C.c_int, [VP, VP, VP]),
    "cgc_grid_set_nlinks": (C.c_int, [VP, C.c_int, VP, VP]),
    "cgc_detect_grid": (C.c_int, [C.c_int32, C.c_int64, VP, VP, P32]),
    "cgc_grid_create_from_edges": (C.c_int, [C.c_int32, C.c_int64, VP, VP, VP, VP, VP, C.POINTER(VP), P32]),
    "cgc_graph_create": (C.c_int, [C.c_int32, C.c_int64, VP, VP, VP, VP, VP, C.POINTER(VP)]),
    "cgc_graph_destroy": (C.c_int, [VP]),
    "cgc_graph_set_tlinks": (C.c_int, [VP, VP, VP]),
    "cgc_graph_maxflow": (C.c_int, [VP, C.POINTER(Options), P64]),
    "cgc_graph_get_segments": (C.c_int, [VP, C.c_int, VP, C.c_uint8, C.c_uint8]),
    "cgc_graph_stats": (C.c_int, [VP, C.POINTER(Stats)]),
    "cgc_grid_set_tlinks_device": (C.c_int, [VP, VP, VP]),
    "cgc_grid_set_nlinks_device": (C.c_int, [VP, C.c_int, VP, VP]),
    "cgc_grid_maxflow": (C.c_int, [VP, C.POINTER(Options), P64]),
    "cgc_grid_maxflow_async": (C.c_int, [VP, C.POINTER(Options)]),
    "cgc_grid_get_labels": (C.c_int, [VP, VP]),
    "cgc_graph_get_state": (C.c_int, [VP, VP, VP]),
    "cgc_grid_wait": (C.c_int, [VP, P64]),
    "cgc_grid_get_segments": (C.c_int, [VP, C.c_int, VP, C.c_uint8, C.c_uint8]),
    "cgc_grid_get_segments_device": (C.c_int, [VP, C.c_int, VP, C.c_uint8, C.c_uint8]),
    "cgc_grid_get_residuals": (C.c_int, [VP, C.POINTER(VP), VP, VP]),
    "cgc_grid_stats": (C.c_int, [VP, C.POINTER(Stats)]),
    "cgc_grid_trace": (C.c_int, [VP, VP, C.c_int32, P32]),
    "cgc_batch_trace": (C.c_int, [VP, VP, C.c_int32, P32]),
    "cgc_grid_maxflow_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, VP, VP, C.POINTER(VP), C.POINTER(VP),
                                           C.POINTER(Options), VP, P64, VP, VP]),
    "cgc_batch_create": (C.c_int, [C.c_int32, VP, VP, C.POINTER(VP)]),
    "cgc_batch_destroy": (C.c_int, [VP]),
    "cgc_batch_set_tlinks": (C.c_int, [VP, C.c_int32, VP, VP]),
    "cgc_batch_set_nlinks": (C.c_int, [VP, C.c_int32, C.c_int, VP, VP]),
    "cgc_batch_maxflow": (C.c_int, [VP, C.POINTER(Options), P64]),
    "cgc_batch_get_segments": (C.c_int, [VP, C.c_int32, C.c_int, VP, C.c_uint8, C.c_uint8]),
    "cgc_batch_stats": (C.c_int, [VP, C.POINTER(Stats)]),
    "cgc_batch_bind_inputs": (C.c_int, [VP, C.c_int32, VP, VP, C.POINTER(VP), C.POINTER(VP)]),
    "cgc_batch_bind_outputs": (C.c_int, [VP, C.c_int32, VP, VP]),
    "cgc_batch_enqueue": (C.c_int, [VP, C.POINTER(Options), VP]),
    "cgc_batch_graph_create": (C.c_int, [VP, C.POINTER(Options), VP]),
    "cgc_batch_graph_launch": (C.c_int, [VP]),
    "cgc_batch_wait": (C.c_int, [VP, P64]),
    "cgc_grid_autotune": (C.c_int, [VP, C.POINTER(Options), C.c_int32, C.c_int32, C.POINTER(Options),
                                    C.POINTER(C.c_double)]),
    "cgc_batch_autotune": (C.c_int, [VP, C.POINTER(Options), C.c_int32, C.c_int32, C.POINTER(Options),
                                     C.POINTER(C.c_double)]),
    "cgc_autotune_lookup": (C.c_int, [C.c_int64, C.c_int32, C.POINTER(Options)]),
    "cgc_scheduler_load": (C.c_int, [VP, VP]),
    "cgc_scheduler_load_file": (C.c_int, [C.c_char_p]),
    "cgc_scheduler_infer": (C.c_int, [C.c_int32, C.c_int32, VP, VP, VP, VP, VP]),
    "cgc_grid_sched_trace": (C.c_int, [VP, VP, VP, VP, C.c_int32, P32]),
    "cgc_trainer_create": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.POINTER(VP)]),
    "cgc_trainer_destroy": (C.c_int, [VP]),
    "cgc_trainer_step": (C.c_int, [VP, C.c_int32, VP, VP, VP, VP, C.c_float, C.c_float, C.POINTER(C.c_float)]),
    "cgc_trainer_eval": (C.c_int, [VP, C.c_int32, VP, VP, VP, VP, C.c_float, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float)]),
    "cgc_trainer_weights": (C.c_int, [VP, VP, VP]),
    "cgc_build_segmentation_graph": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, VP, VP, C.c_float, C.c_int32,
                                               C.c_int32, C.c_int32, VP, VP, VP, VP, VP, VP]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads libcgc.so once; raises if it is absent (build it with
    `python -m cugip_b200.build` or `__graft_entry__.build()`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libcgc.so not built: {path} is missing (run cugip_b200/build.py)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != CGC_OK:
        raise CgcError(rc, load().cgc_last_error().decode(errors="replace"))


OPTION_FIELDS = ("local_pulses", "sweeps_per_relabel", "wait_limit_us", "max_sweeps", "persistent",
                 "region_relabels", "stall_sweeps", "ctas_per_sm", "learned", "trace_cycles", "bfs_warp_min",
                 "exclusive", "relabel")


def options(**fields) -> Options:
    """A cgc_options with struct_size set; fields left out are 0 (the default)."""
    o = Options()
    o.struct_size = C.sizeof(Options)
    for k, v in fields.items():
        if k not in OPTION_FIELDS:
            raise TypeError(f"unknown option {k!r}")
        setattr(o, k, int(v))
    return o
