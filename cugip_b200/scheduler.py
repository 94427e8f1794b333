"""Learned tile scheduler: traces from plain solves, training with the
library's own CUDA kernels (cgc_trainer_*), and the weight file.

Training data: plain solves of 128^3 instances of the two-sphere generator
(workload 5, instances 0..n-1) run with `TRACE_POLICY`; for each of the first
relabel cycles the solve records every tile's 10 features and, as labels,
whether the tile delivered flow to the sink during the cycle (priority) and
the last pulse of its first visit that moved flow out of the tile or into the
sink, up to 32 (budget).  Only tiles active
at the start of the cycle count in the loss.

    python -m cugip_b200.scheduler --solves 2000      # writes scheduler_weights.bin
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import struct
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib, volume
from ._lib import check
from .graph_cut import GridGraph, Policy

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "scheduler_weights.bin")
MAGIC = b"CGCSCHD1"
NCONV = 3 * 27 * 16 * 16
NHEAD = 2 * 16 + 2
# traces come from the plain production schedule
TRACE_POLICY = Policy(local_pulses=4, region_relabels=2, sweeps_per_relabel=8, trace_cycles=4)


def save_weights(path: str, conv_bf16: np.ndarray, head: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.ascontiguousarray(conv_bf16, dtype=np.uint16).tobytes())
        f.write(np.ascontiguousarray(head, dtype=np.float32).tobytes())


def load_weights(path: str = WEIGHTS) -> None:
    """Loads the scheduler weights into the library (needed before Policy(learned=1))."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"no scheduler weights at {path} (train with python -m cugip_b200.scheduler)")
    check(_lib.load().cgc_scheduler_load_file(path.encode()))


def collect(n: int, first_index: int = 0, threads: int = 4, log_every: int = 200):
    """Runs n plain traced solves; returns (features uint16 [M,T,16], pulses uint8 [M,T], sink uint8 [M,T])."""
    spec0 = volume.preset(5, first_index)
    g = GridGraph(spec0.X, spec0.Y, spec0.Z)
    feats, pulses, sinks = [], [], []
    t0 = time.time()
    with ThreadPoolExecutor(max_workers=threads) as pool:   # generation runs in C, outside the GIL
        futs = [pool.submit(volume.workload, 5, first_index + k) for k in range(min(n, 2 * threads))]
        for k in range(n):
            v = futs[k].result()
            futs[k] = None
            if k + 2 * threads < n:
                futs.append(pool.submit(volume.workload, 5, first_index + k + 2 * threads))
            g.set_tweights(v.capS, v.capT)
            for ax in range(3):
                g.set_nweights(ax, v.n[ax])
            g.max_flow(TRACE_POLICY)
            f, p, s = g.sched_trace()
            feats.append(f)
            pulses.append(p)
            sinks.append(s)
            if log_every and (k + 1) % log_every == 0:
                print(f"  traced {k + 1}/{n} solves ({time.time() - t0:.1f} s)", flush=True)
    g.close()
    return np.concatenate(feats), np.concatenate(pulses), np.concatenate(sinks)


def train(feats: np.ndarray, pulses: np.ndarray, sinks: np.ndarray, epochs: int = 6, batch: int = 16,
          lr: float = 2e-3, seed: int = 0, val_frac: float = 0.1, log=print):
    """Trains with cgc_trainer_step on the GPU; returns (conv_bf16, head, history)."""
    import torch
    lib = _lib.load()
    M, T, _ = feats.shape
    D = round(T ** (1 / 3))
    assert D ** 3 == T
    dev = torch.device("cuda")
    F = torch.from_numpy(feats.astype(np.int16)).to(dev)                      # BF16 bits
    active = F.view(torch.bfloat16)[:, :, 1].float() > 0
    mask = active.float().contiguous()
    yprio = torch.from_numpy(sinks.astype(np.float32)).to(dev)
    # budget label: productive pulses of the first visit (0 = not visited and
    # 255 = moved nothing out of the tile both mean one pulse)
    pl = pulses.astype(np.float32)
    pl[(pulses == 0) | (pulses == 255)] = 1.0
    ybud = (torch.from_numpy(pl).to(dev).clamp(1, 32) - 1) / 31.0
    rng = np.random.default_rng(seed)
    order = rng.permutation(M)
    nval = max(1, int(M * val_frac))
    val, tr_idx = order[:nval], order[nval:]
    h = C.c_void_p()
    check(lib.cgc_trainer_create(batch, D, seed, C.byref(h)))
    history = []

    def run(idx, step):
        loss = C.c_float()
        acc = C.c_float()
        sel = torch.from_numpy(np.asarray(idx)).to(dev)
        f, p, b, m = F[sel].contiguous(), yprio[sel].contiguous(), ybud[sel].contiguous(), mask[sel].contiguous()
        cnt = float(m.sum().item())
        if cnt == 0:
            return None, None
        if step:
            check(lib.cgc_trainer_step(h, len(idx), f.data_ptr(), p.data_ptr(), b.data_ptr(), m.data_ptr(), cnt,
                                       lr, C.byref(loss)))
            return loss.value, None
        check(lib.cgc_trainer_eval(h, len(idx), f.data_ptr(), p.data_ptr(), b.data_ptr(), m.data_ptr(), cnt,
                                   C.byref(loss), C.byref(acc)))
        return loss.value, acc.value

    try:
        for ep in range(epochs):
            rng.shuffle(tr_idx)
            tl = [run(tr_idx[i:i + batch], True)[0] for i in range(0, len(tr_idx) - batch + 1, batch)]
            tl = [x for x in tl if x is not None]
            vl, va = [], []
            for i in range(0, len(val), batch):
                l_, a_ = run(val[i:i + batch], False)
                if l_ is not None:
                    vl.append(l_)
                    va.append(a_)
            rec = {"epoch": ep, "train_loss": float(np.mean(tl)) if tl else None,
                   "val_loss": float(np.mean(vl)) if vl else None, "val_prio_acc": float(np.mean(va)) if va else None}
            history.append(rec)
            log(f"  epoch {ep}: {rec}")
        conv = np.zeros(NCONV, np.uint16)
        head = np.zeros(NHEAD, np.float32)
        check(lib.cgc_trainer_weights(h, conv.ctypes.data, head.ctypes.data))
    finally:
        lib.cgc_trainer_destroy(h)
    return conv, head, history


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--solves", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--threads", type=int, default=max(1, min(8, (os.cpu_count() or 2) // 4)))
    args = ap.parse_args()
    check(_lib.load().cgc_init(0))
    t0 = time.time()
    feats, pulses, sinks = collect(args.solves, threads=args.threads)
    print(f"traces: {feats.shape[0]} relabel cycles x {feats.shape[1]} tiles from {args.solves} solves "
          f"in {time.time() - t0:.1f} s", flush=True)
    conv, head, hist = train(feats, pulses, sinks, epochs=args.epochs, batch=args.batch, lr=args.lr)
    save_weights(args.out, conv, head)
    print(f"wrote {args.out}; final {hist[-1]}")


if __name__ == "__main__":
    main()
