"""Device-side graph construction from image + markers (the reference's
segmentation front-end) and the segmentation entry points."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def numpy_build(img, mk, sigma, scale, hard, gaussian=False):
    """CPU restatement of benchmarks/graph_cut/graph_cut.cpp:56-79 in float32."""
    Z, Y, X = img.shape
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    capS = np.where(mk == 128, hard, 0).astype(np.int32)
    capT = np.where(mk == 255, hard, 0).astype(np.int32)
    lo = np.minimum(np.minimum(x, y), z)
    hi = np.minimum(np.minimum(X - x, Y - y), Z - z)
    border = (lo <= 1) | (hi <= 2)
    capS[border] = hard
    capT[border] = 0
    s2 = np.float32(sigma) * np.float32(sigma)
    out = []
    for axnp in (2, 1, 0):
        n = np.zeros_like(capS)
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[axnp] = slice(0, -1)
        b[axnp] = slice(1, None)
        d = img[tuple(a)] - img[tuple(b)]
        q = (d * d) / np.float32(2.0) / s2 if gaussian else (d * d) / np.float32(2.0) * s2
        n[tuple(a)] = np.floor(np.float32(scale) * np.exp(-q).astype(np.float32) + np.float32(0.5)).astype(np.int32)
        out.append(n)
    return capS, capT, out


def scene(seed, shape=(20, 30, 40)):
    rng = np.random.default_rng(seed)
    Z, Y, X = shape
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    blob = ((x - X / 2) ** 2 / (X / 4) ** 2 + (y - Y / 2) ** 2 / (Y / 4) ** 2 + (z - Z / 2) ** 2 / (Z / 4) ** 2) < 1
    img = (0.2 + 0.6 * blob + rng.normal(0, 0.05, shape)).astype(np.float32)
    mk = np.zeros(shape, np.uint8)
    mk[Z // 2, Y // 2, X // 2 - 2: X // 2 + 2] = 255
    mk[3, 3:6, 3:6] = 128
    return img, mk


@pytest.mark.parametrize("gaussian,sigma", [(False, 1.0), (False, 3.0), (True, 0.1)])
def test_device_build_matches_the_front_end(gaussian, sigma):
    import torch
    from cugip_b200.segment import build_graph
    img, mk = scene(1)
    caps = [c.cpu().numpy() for c in build_graph(img, mk, sigma, 1000, 1_000_000, gaussian)]
    ref = numpy_build(img, mk, sigma, 1000, 1_000_000, gaussian)
    assert np.array_equal(caps[0], ref[0]) and np.array_equal(caps[1], ref[1])
    for a in range(3):
        diff = np.abs(caps[2 + a].astype(np.int64) - ref[2][a])
        # expf on the GPU and numpy's float32 exp may differ by an ulp, which
        # can move a value across a rounding boundary
        assert diff.max() <= 1 and (diff > 0).mean() < 1e-3


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_segmentation_is_exact_on_the_built_graph(seed):
    from cugip_b200 import _lib
    from cugip_b200.graph_cut import SOURCE
    from cugip_b200.segment import build_graph, segment
    _lib.check(_lib.load().cgc_init(0))
    img, mk = scene(seed)
    Z, Y, X = img.shape
    sigma = 3.0 if seed != 2 else 0.1
    gaussian = seed == 2
    caps = [c.cpu().numpy().reshape(-1) for c in build_graph(img, mk, sigma, gaussian=gaussian)]
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, caps[0], caps[1], caps[2:])
    mask, flow = segment(img, mk, sigma, mask_value=255, gaussian=gaussian)
    assert flow == f0
    assert np.array_equal(mask.reshape(-1), t0 * 255)
    mask_s, _ = segment(img, mk, sigma, mask_value=1, which=SOURCE, gaussian=gaussian)
    assert np.array_equal(mask_s.reshape(-1), s0)
    assert mask[Z // 2, Y // 2, X // 2] == 255  # sink markers are on the mask side
