"""Synthetic capacity volumes (wraps cgc_volume_preset / cgc_volume_generate).

Workloads: 1 = 64^3 two spheres, 2 = 256^3 forty spheres, 3 = 512x512x128
two hundred tubes, 4 = batched instance `index` (extents 32..160),
5 = 128^3 training instance `index`.  All capacities are int32, x-fastest.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check


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


def preset(which: int, index: int = 0) -> _lib.VolumeSpec:
    spec = _lib.VolumeSpec()
    check(_lib.load().cgc_volume_preset(int(which), int(index), C.byref(spec)))
    return spec


def generate(spec: _lib.VolumeSpec, with_image: bool = False) -> Volume:
    N = spec.X * spec.Y * spec.Z
    capS = np.empty(N, np.int32)
    capT = np.empty(N, np.int32)
    n = [np.empty(N, np.int32) for _ in range(3)]
    img = np.empty(N, np.float32) if with_image else None
    ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
    check(_lib.load().cgc_volume_generate(C.byref(spec), ptr(capS), ptr(capT), ptr(n[0]), ptr(n[1]), ptr(n[2]),
                                          ptr(img)))
    return Volume(spec.X, spec.Y, spec.Z, capS, capT, n, img)


def workload(which: int, index: int = 0, **overrides) -> Volume:
    spec = preset(which, index)
    for k, v in overrides.items():
        setattr(spec, k, v)
    return generate(spec)
