"""Builds libcgc.so (the CUDA engine + C ABI) in-tree for sm_100a.

The library is compiled with nvcc directly (no JIT cache), so the built file
sits next to this module and travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libcgc.so")
# the same engine with every tile / neighbour / worklist index checked (CGC_BOUNDS_CHECK)
BOUNDS_LIB = os.path.join(HERE, "libcgc_bounds.so")
# synthetic workloads: host code only, so that CPU-only callers need no CUDA library
VOL_LIB = os.path.join(HERE, "libcgcvol.so")
VOL_SOURCES = ["cgc_volume.cpp"]

SOURCES = ["cgc_engine.cu", "cgc_batch.cu", "cgc_autotune.cu", "cgc_sched_train.cu", "cgc_noalloc.cu",
           "cgc_build.cu", "cgc_csr.cu", "cgc_graph.cpp"]
HEADERS = ["cgc_device.cuh", "cgc_kernels.cuh", "cgc_internal.h", "cgc_pool.h", "cgc_sched.cuh",
           "cgc_sync.cuh", "cgc_warp.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-fopenmp",
    "-shared", "-lgomp",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_volume(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in VOL_SOURCES] + [os.path.join(INCLUDE, "cgc_volume.h"),
                                                            os.path.join(INCLUDE, "cgc.h"), __file__]
    if not force and not _stale(VOL_LIB, deps):
        return VOL_LIB
    cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-fopenmp", "-I", INCLUDE, "-o", VOL_LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in VOL_SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(VOL_LIB + ".tmp", VOL_LIB)
    return VOL_LIB


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None, bounds_check: bool = False) -> str:
    """Builds libcgc.so (or, with bounds_check, libcgc_bounds.so: the same
    sources with -DCGC_BOUNDS_CHECK, for test runs only)."""
    build_volume(force, verbose)
    lib = BOUNDS_LIB if bounds_check else LIB
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(INCLUDE, "cgc.h"), __file__]
    if not force and not _stale(lib, deps):
        return lib
    flags = ["-DCGC_BOUNDS_CHECK"] if bounds_check else []
    cmd = [_nvcc(), *NVCC_FLAGS, *flags, *(extra or []), "-I", INCLUDE, "-I", CSRC, "-o", lib + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True,
                extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None,
                bounds_check="--bounds-check" in sys.argv))
