"""C ABI surface without a GPU: the library loads, exports every entry point
that include/cgc.h declares, and its host-only logic behaves."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from cugip_b200 import _lib
from cugip_b200.graph_cut import GridGraph, _i32
from tests import graphs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "cgc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cgc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_volume_library_is_host_only_and_exports_its_header():
    """libcgcvol.so (the synthetic workloads) exports every function of
    include/cgc_volume.h and links no CUDA library, so the CPU baseline can
    build workloads without the GPU engine."""
    from cugip_b200 import volume
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "cgc_volume.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(cgc_[a-z0-9_]+)\s*\(", text)))
    lib = volume.load()
    assert names == ["cgc_volume_generate", "cgc_volume_last_error", "cgc_volume_preset"]
    for name in names:
        assert hasattr(lib, name), name
    import subprocess
    deps = subprocess.run(["ldd", volume.VOL_LIB_PATH], capture_output=True, text=True).stdout
    assert "libcuda" not in deps and "libcudart" not in deps, deps
    with pytest.raises(_lib.CgcError):
        volume.preset(99)


def test_no_device_is_reported_not_hidden():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    assert lib.cgc_init(0) == 9  # CGC_ERR_NO_DEVICE
    with pytest.raises(_lib.CgcError):
        GridGraph(8, 8, 8)


def detect(n, a, b):
    dims = (C.c_int32 * 3)()
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    rc = _lib.load().cgc_detect_grid(n, a.size, a.ctypes.data, b.ctypes.data, dims)
    return rc, tuple(dims)


def test_detect_grid_on_reference_four_by_four():
    n, a, b, *_ = graphs.four_by_four()
    rc, dims = detect(n, a, b)
    assert rc == 0 and dims == (4, 4, 1)


@pytest.mark.parametrize("dims", [(7, 5, 3), (16, 16, 4), (9, 1, 1), (1, 9, 1), (1, 1, 9), (12, 10, 1), (5, 1, 6)])
def test_detect_grid_random(dims):
    X, Y, Z = dims
    _, _, fwd, bwd = graphs.random_grid(X, Y, Z, 3)
    a, b, _, _ = graphs.grid_edges(X, Y, Z, fwd, bwd)
    rc, got = detect(X * Y * Z, a, b)
    assert rc == 0
    # any factorisation that maps every edge to a grid edge is the same graph
    gx, gy, gz = got
    assert gx * gy * gz == X * Y * Z
    assert got == dims or (X, Y, Z).count(1) >= 1


def test_detect_grid_rejects_non_grids():
    n, a, b, *_ = graphs.layered(layers=4, size=16, nbrs=3)
    rc, _ = detect(n, a, b)
    assert rc == 8  # CGC_ERR_NOT_GRID
    rc, _ = detect(10, [0, 1], [5, 5])  # row-wrapping step
    assert rc in (0, 8)
    rc, _ = detect(4, [0], [0])  # self loop
    assert rc == 8


def test_capacity_validation_happens_before_the_device():
    with pytest.raises(_lib.CgcError):
        _i32(np.array([1.5, 2.0]), 2, "x")
    with pytest.raises(_lib.CgcError):
        _i32(np.array([-1, 2]), 2, "x")
    with pytest.raises(_lib.CgcError):
        _i32(np.array([1, 2, 3]), 2, "x")
    assert _i32(np.array([1.0, 2.0]), 2, "x").dtype == np.int32


def test_volume_presets():
    from cugip_b200 import volume
    s = volume.preset(1)
    assert (s.X, s.Y, s.Z, s.count) == (64, 64, 64, 2)
    s = volume.preset(3)
    assert (s.X, s.Y, s.Z, s.kind) == (512, 512, 128, 1)
    for i in range(20):
        s = volume.preset(4, i)
        assert 32 <= s.X <= 160 and 32 <= s.Y <= 160 and 32 <= s.Z <= 160 and 4 <= s.count <= 20
    with pytest.raises(_lib.CgcError):
        volume.preset(9)
