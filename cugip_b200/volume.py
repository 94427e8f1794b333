"""Synthetic capacity volumes (wraps cgc_volume_preset / cgc_volume_generate of
libcgcvol.so, a host-only library: building a workload loads no CUDA code).

Workloads: 1 = 64^3 two spheres, 2 = 256^3 forty spheres, 3 = 512x512x128
two hundred tubes, 4 = batched instance `index` (extents 32..160),
5 = 128^3 training instance `index`.  All capacities are int32, x-fastest.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from ._lib import CgcError

VOL_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcgcvol.so")


class VolumeSpec(C.Structure):
    _fields_ = [("X", C.c_int32), ("Y", C.c_int32), ("Z", C.c_int32), ("kind", C.c_int32),
                ("seed", C.c_uint64), ("count", C.c_int32), ("n_fixed_radii", C.c_int32),
                ("fixed_radii", C.c_double * 8), ("radius_min", C.c_double), ("radius_max", C.c_double),
                ("intensity_min", C.c_double), ("intensity_max", C.c_double), ("background", C.c_double),
                ("noise_sd", C.c_double), ("mu_bg", C.c_double), ("mu_fg", C.c_double), ("class_sd", C.c_double),
                ("tlink_scale", C.c_double), ("nlink_scale", C.c_double), ("nlink_sigma", C.c_double),
                ("ctrl_min", C.c_int32), ("ctrl_max", C.c_int32), ("edge_sigma", C.c_double)]


_vol = None


def load() -> C.CDLL:
    """Loads libcgcvol.so once; raises if it is absent (cugip_b200/build.py builds it)."""
    global _vol
    if _vol is None:
        if not os.path.exists(VOL_LIB_PATH):
            raise RuntimeError(f"libcgcvol.so not built: {VOL_LIB_PATH} is missing (run cugip_b200/build.py)")
        lib = C.CDLL(VOL_LIB_PATH)
        lib.cgc_volume_preset.restype = C.c_int
        lib.cgc_volume_preset.argtypes = [C.c_int, C.c_int32, C.POINTER(VolumeSpec)]
        lib.cgc_volume_generate.restype = C.c_int
        lib.cgc_volume_generate.argtypes = [C.POINTER(VolumeSpec)] + [C.c_void_p] * 6
        lib.cgc_volume_last_error.restype = C.c_char_p
        lib.cgc_volume_last_error.argtypes = []
        _vol = lib
    return _vol


def check(rc: int) -> None:
    if rc != 0:
        raise CgcError(rc, load().cgc_volume_last_error().decode(errors="replace"))


@dataclass
class Volume:
    X: int
    Y: int
    Z: int
    capS: np.ndarray   # (N,) int32 source t-links
    capT: np.ndarray   # (N,) int32 sink t-links
    n: list            # 3 x (N,) int32 symmetric n-links to +x, +y, +z
    image: np.ndarray | None = None

    @property
    def N(self) -> int:
        return self.X * self.Y * self.Z

    def arrays(self):
        return self.capS, self.capT, self.n[0], self.n[1], self.n[2]


def preset(which: int, index: int = 0) -> VolumeSpec:
    spec = VolumeSpec()
    check(load().cgc_volume_preset(int(which), int(index), C.byref(spec)))
    return spec


def generate(spec: VolumeSpec, with_image: bool = False) -> Volume:
    N = spec.X * spec.Y * spec.Z
    capS = np.empty(N, np.int32)
    capT = np.empty(N, np.int32)
    n = [np.empty(N, np.int32) for _ in range(3)]
    img = np.empty(N, np.float32) if with_image else None
    ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
    check(load().cgc_volume_generate(C.byref(spec), ptr(capS), ptr(capT), ptr(n[0]), ptr(n[1]), ptr(n[2]),
                                          ptr(img)))
    return Volume(spec.X, spec.Y, spec.Z, capS, capT, n, img)


def workload(which: int, index: int = 0, **overrides) -> Volume:
    spec = preset(which, index)
    for k, v in overrides.items():
        setattr(spec, k, v)
    return generate(spec)
