"""Segmentation front-end: image + markers -> grid graph on the device -> exact
max-flow -> mask, mirroring the reference's `computeCudaGraphCut`
(benchmarks/graph_cut/graph_cut.cpp:33-98) and its `grid_segmentation` command
line (benchmarks/graph_cut/segmentation.cpp:79-239).  The reference reads ITK
images; here the command line reads raw volumes (x fastest).

    python -m cugip_b200.segment -i image.f32 -m markers.u8 --dims X Y Z -s 1.0 -o mask.u8 [-v 255]

The mask marks the voxels that can reach the sink (marker 255) side, as the
reference's Graph::fill_segments does (graph_cut.hpp:304-333).
"""
from __future__ import annotations

import argparse

import numpy as np

from . import _lib
from ._lib import check
from .graph_cut import SINK, SOURCE, GridGraph, Policy


def build_graph(image, markers, sigma: float, nlink_scale: int = 1000, hard_tlink: int = 1_000_000,
                gaussian: bool = False):
    """Device capacity volumes (torch int32 tensors, x fastest): capS, capT, nx, ny, nz.
    `image` / `markers`: arrays of shape (Z, Y, X) (numpy or CUDA tensors)."""
    import torch
    img = torch.as_tensor(np.asarray(image, np.float32) if not torch.is_tensor(image) else image,
                          dtype=torch.float32).cuda().contiguous()
    Z, Y, X = img.shape
    mk = None
    if markers is not None:
        mk = torch.as_tensor(np.asarray(markers, np.uint8) if not torch.is_tensor(markers) else markers,
                             dtype=torch.uint8).cuda().contiguous()
        if tuple(mk.shape) != (Z, Y, X):
            raise ValueError("markers must have the image's shape")
    caps = [torch.empty((Z, Y, X), dtype=torch.int32, device=img.device) for _ in range(5)]
    check(_lib.load().cgc_build_segmentation_graph(
        X, Y, Z, img.data_ptr(), mk.data_ptr() if mk is not None else None, float(sigma), int(nlink_scale),
        int(hard_tlink), 1 if gaussian else 0, *[c.data_ptr() for c in caps], None))
    return caps


def segment(image, markers, sigma: float = 1.0, mask_value: int = 255, background: int = 0,
            nlink_scale: int = 1000, hard_tlink: int = 1_000_000, gaussian: bool = False,
            policy: Policy | None = None, which: str = SINK):
    """Returns (mask of shape (Z, Y, X), flow)."""
    import torch
    caps = build_graph(image, markers, sigma, nlink_scale, hard_tlink, gaussian)
    Z, Y, X = caps[0].shape
    g = GridGraph(X, Y, Z)
    try:
        g.set_tweights_device(caps[0].data_ptr(), caps[1].data_ptr())
        for ax in range(3):
            g.set_nweights_device(ax, caps[2 + ax].data_ptr())
        flow = g.max_flow(policy)
        out = torch.empty((Z, Y, X), dtype=torch.uint8, device=caps[0].device)
        g.fill_segments_device(out.data_ptr(), mask_value, background, which)
        return out.cpu().numpy(), flow
    finally:
        g.close()


def main():
    ap = argparse.ArgumentParser(description="grid graph-cut segmentation (exact max-flow on the GPU)")
    ap.add_argument("-i", "--input", required=True, help="raw float32 image, x fastest")
    ap.add_argument("-m", "--markers", required=True, help="raw uint8 markers (128 = source, 255 = sink)")
    ap.add_argument("-o", "--output", required=True, help="raw uint8 mask")
    ap.add_argument("--dims", type=int, nargs=3, required=True, metavar=("X", "Y", "Z"))
    ap.add_argument("-s", "--sigma", type=float, default=1.0)
    ap.add_argument("-v", "--mask-value", type=int, default=255)
    ap.add_argument("--nlink-scale", type=int, default=1000)
    ap.add_argument("--hard", type=int, default=1_000_000)
    ap.add_argument("--gaussian", action="store_true", help="exp(-d^2/(2 sigma^2)) instead of the reference formula")
    args = ap.parse_args()
    X, Y, Z = args.dims
    img = np.fromfile(args.input, dtype=np.float32).reshape(Z, Y, X)
    mk = np.fromfile(args.markers, dtype=np.uint8).reshape(Z, Y, X)
    check(_lib.load().cgc_init(0))
    mask, flow = segment(img, mk, args.sigma, args.mask_value, nlink_scale=args.nlink_scale, hard_tlink=args.hard,
                         gaussian=args.gaussian)
    mask.tofile(args.output)
    print(f"max flow {flow}; {int((mask == args.mask_value).sum())} voxels marked")


if __name__ == "__main__":
    main()
