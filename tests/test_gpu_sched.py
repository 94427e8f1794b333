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


def test_trainer_learns_a_synthetic_target_and_inference_agrees():
    """cgc_trainer_step (tensor-core forward, FP32 backward, Adam) on a learnable
    target -- priority = (feature 0 of the tile > 0.5), budget = feature 1 --
    lowers the loss, and the trained weights run through the solve's inference
    kernels (cgc_scheduler_infer) reproduce the priorities on the active tiles."""
    import torch
    lib = _lib.load()
    D, grids, steps = 8, 8, 300
    T = D ** 3
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", 0)

    def batch():
        f = np.zeros((grids, T, 16), np.float32)
        act = rng.random((grids, T)) < 0.4
        f[..., :10] = rng.random((grids, T, 10)) * act[..., None]
        f = torch.from_numpy(f).to(torch.bfloat16)
        fv = f.float().numpy()
        prio = ((fv[..., 0] > 0.5) & act).astype(np.float32)
        bud = np.clip(fv[..., 1], 0, 1).astype(np.float32)
        return f.view(torch.int16).to(dev).contiguous(), torch.from_numpy(prio).to(dev), \
            torch.from_numpy(bud).to(dev), torch.from_numpy(act.astype(np.float32)).to(dev), act, fv

    h = C.c_void_p()
    _lib.check(lib.cgc_trainer_create(grids, D, 11, C.byref(h)))
    try:
        ev = batch()
        loss0, acc0 = C.c_float(), C.c_float()
        _lib.check(lib.cgc_trainer_eval(h, grids, ev[0].data_ptr(), ev[1].data_ptr(), ev[2].data_ptr(), ev[3].data_ptr(),
                                        float(ev[4].sum()), C.byref(loss0), C.byref(acc0)))
        loss = C.c_float()
        for _ in range(steps):
            b = batch()
            _lib.check(lib.cgc_trainer_step(h, grids, b[0].data_ptr(), b[1].data_ptr(), b[2].data_ptr(), b[3].data_ptr(),
                                            float(b[4].sum()), 3e-3, C.byref(loss)))
        loss1, acc1 = C.c_float(), C.c_float()
        _lib.check(lib.cgc_trainer_eval(h, grids, ev[0].data_ptr(), ev[1].data_ptr(), ev[2].data_ptr(), ev[3].data_ptr(),
                                        float(ev[4].sum()), C.byref(loss1), C.byref(acc1)))
        assert loss1.value < 0.6 * loss0.value, (loss0.value, loss1.value)
        assert acc1.value > 0.85, acc1.value
        conv = np.zeros(3 * 27 * 256, np.uint16)
        head = np.zeros(34, np.float32)
        _lib.check(lib.cgc_trainer_weights(h, conv.ctypes.data, head.ctypes.data))
    finally:
        lib.cgc_trainer_destroy(h)
    _lib.check(lib.cgc_scheduler_load(conv.ctypes.data, head.ctypes.data))
    budget = torch.zeros(grids * T, dtype=torch.uint8, device=dev)
    prio = torch.zeros(grids * T, dtype=torch.uint8, device=dev)
    _lib.check(lib.cgc_scheduler_infer(grids, D, ev[0].data_ptr(), budget.data_ptr(), prio.data_ptr(), None, None))
    act = ev[4].reshape(-1)
    want = (ev[5][..., 0] > 0.5).reshape(-1)
    got = prio.cpu().numpy().astype(bool)
    assert (got[act] == want[act]).mean() > 0.85
