"""The learned scheduler's CNN on the tensor cores (cgc_scheduler_infer, the
kernels the solve runs after every global relabel) against a plain PyTorch
fp32 reference of the same network: three bias-free 3x3x3 convolutions with
16 channels, ReLU, BF16 weights and activations (rounded between layers, as
the kernels store them), then the linear head.

Tolerance: the kernels accumulate in FP32 in another order than torch, so an
activation can round to the neighbouring BF16 value; the head logits agree to
2e-2 absolute on 99 % of the tiles, the budgets (1..32) to +-1 on 99 % and the
priorities on 99 % (they differ only where a logit is within rounding of 0)."""
import ctypes as C

import numpy as np
import pytest

from cugip_b200 import _lib

pytestmark = pytest.mark.gpu


def _random_weights(seed):
    rng = np.random.default_rng(seed)
    w = (rng.standard_normal((3, 27, 16, 16)) * np.sqrt(2.0 / (27 * 16))).astype(np.float32)
    head = np.zeros(34, np.float32)
    head[:32] = rng.standard_normal(32) * 0.5
    head[32:] = [0.1, -0.2]
    return w, head


def _bf16_bits(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).view(torch.int16).numpy().view(
        np.uint16)


def _reference(feat, w, head, grids, D):
    """torch fp32: feat (grids, D, D, D, 16) -> logits (grids*D^3, 2)."""
    import torch
    x = torch.from_numpy(feat).permute(0, 4, 1, 2, 3).contiguous()  # N, C, z, y, x
    for layer in range(3):
        # tap k = (dx+1) + 3(dy+1) + 9(dz+1); W[layer][k][cin][cout] -> weight[cout][cin][dz][dy][dx]
        wt = torch.from_numpy(w[layer].reshape(3, 3, 3, 16, 16)).permute(4, 3, 0, 1, 2).contiguous()
        x = torch.nn.functional.conv3d(x, wt, padding=1).clamp_min(0)
        x = x.to(torch.bfloat16).float()
    a = x.permute(0, 2, 3, 4, 1).reshape(-1, 16)
    hw = torch.from_numpy(head)
    p0 = a @ hw[:16] + hw[32]
    p1 = a @ hw[16:32] + hw[33]
    return torch.stack([p0, p1], 1).numpy()


@pytest.mark.parametrize("grids,D,seed", [(2, 8, 1), (1, 16, 2), (3, 5, 3)])
def test_tensor_core_cnn_matches_fp32_reference(grids, D, seed):
    import torch
    lib = _lib.load()
    w, head = _random_weights(seed)
    wb = _bf16_bits(w.reshape(-1))
    wf = torch.from_numpy(w).to(torch.bfloat16).float().numpy()  # the weights as the kernels see them
    _lib.check(lib.cgc_scheduler_load(wb.ctypes.data, head.ctypes.data))
    rng = np.random.default_rng(100 + seed)
    feat = np.zeros((grids, D, D, D, 16), np.float32)
    active = rng.random((grids, D, D, D)) < 0.3  # inactive tiles keep all-zero features
    feat[..., :10] = rng.random((grids, D, D, D, 10)) * active[..., None]
    feat = torch.from_numpy(feat).to(torch.bfloat16).float().numpy()
    T = grids * D ** 3
    dev = torch.device("cuda", 0)
    d_feat = torch.from_numpy(_bf16_bits(feat.reshape(-1)).view(np.int16)).to(dev)
    budget = torch.zeros(T, dtype=torch.uint8, device=dev)
    prio = torch.zeros(T, dtype=torch.uint8, device=dev)
    logits = torch.zeros(2 * T, dtype=torch.float32, device=dev)
    _lib.check(lib.cgc_scheduler_infer(grids, D, d_feat.data_ptr(), budget.data_ptr(), prio.data_ptr(),
                                       logits.data_ptr(), None))
    got = logits.cpu().numpy().reshape(T, 2)
    ref = _reference(feat, wf, head, grids, D)
    close = np.abs(got - ref) <= 2e-2 + 2e-2 * np.abs(ref)
    assert close.all(axis=1).mean() >= 0.99, np.abs(got - ref).max()
    ref_budget = np.clip(1 + np.floor(31.0 / (1.0 + np.exp(-ref[:, 1])) + 0.5), 1, 32)
    assert (np.abs(budget.cpu().numpy().astype(np.int64) - ref_budget) <= 1).mean() >= 0.99
    assert ((prio.cpu().numpy() == 1) == (ref[:, 0] >= 0)).mean() >= 0.99
    # an all-zero grid gives exactly the biases
    d_feat.zero_()
    _lib.check(lib.cgc_scheduler_infer(grids, D, d_feat.data_ptr(), budget.data_ptr(), prio.data_ptr(),
                                       logits.data_ptr(), None))
    z = logits.cpu().numpy().reshape(T, 2)
    assert np.array_equal(z[:, 0], np.full(T, head[32], np.float32))
    assert np.array_equal(z[:, 1], np.full(T, head[33], np.float32))
