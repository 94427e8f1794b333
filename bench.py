#!/usr/bin/env python
"""Benchmark: voxels/s to the exact max flow (plus both cut sets) on a grid.

A step is one full solve of the 256^3 forty-sphere workload (16.7 M voxels,
50 M n-links, int32 capacities): capacities -> exact int64 flow, the minimal
source set and the sink-reachable set, all checked against the oracle's
golden answer after the timed region.

  value : the production path -- device-resident capacities bound to a
          one-instance batch, the solve captured in a CUDA graph and replayed
          once per step, masks written to device memory; the schedule is the
          autotuner's choice among plain and learned-scheduler candidates.
          Whole-job voxels/s over all ranks (each rank solves its own replica:
          a single grid does not shard).
  e2e   : the same step through the host API (GridGraph.set_tweights /
          set_nweights from pinned host arrays, both masks copied back to the
          host), copies inside the timing; two grids on two streams so that
          one step's uploads overlap the previous step's solve (the serial
          one-grid figure is reported beside it).
  variants : plain fixed-schedule single solves vs tuned vs learned, on the
          256^3 grid and on the 96-instance batch (extents 32..160): plain
          sequential solves vs one batched graph launch vs learned + batched.

`--impl reference` times the CPU max-flow path (the oracle's Boykov-Kolmogorov
restatement of the reference's BK call site) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {1: "grid 64^3 two Gaussian spheres", 2: "grid 256^3 forty Gaussian spheres",
             3: "grid 512x512x128 two hundred tubes"}
METRIC = "voxels/s to exact max-flow (flow value + canonical cut), 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", type=int, default=2, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--batch-instances", type=int, default=96)
    ap.add_argument("--schedule", default="",
                    help="fixed schedule L,R,K,ctas,learned (skips the autotuner; for profiling)")
    return ap.parse_args()


def golden(workload: int, index: int = 0):
    try:
        g = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))
        for c in g["cases"]:
            if c["workload"] == workload and c["index"] == index:
                return c
    except Exception:
        pass
    return None


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


LEARNED_MODES = {1: "budgets + priorities in throughput-bound cycles", 2: "budgets only, throughput-bound cycles",
                 3: "budgets in every cycle + priorities in throughput-bound cycles"}


def learned_report(workloads=(1, 2, 3)) -> dict:
    """The learned scheduler (each mode) against the same fixed schedule without
    it, on the 64^3 two-sphere, 256^3 forty-sphere and 512x512x128 tube
    workloads: kernel time, time in the scheduler stage, sweeps, exact global
    relabels (saved = plain - learned), tile visits, pulses and bit-identity of
    the flow and of both cut sets."""
    import hashlib
    import torch
    from cugip_b200 import volume
    from cugip_b200.graph_cut import SINK, SOURCE, GridGraph, Policy
    base = dict(local_pulses=4, region_relabels=2, sweeps_per_relabel=8, ctas_per_sm=3)
    keep = ("kernel_ms", "sched_ms", "sweeps", "global_relabels", "tiles_swept", "pulses")
    out = {}
    for w in workloads:
        v = volume.workload(w)
        d = [torch.from_numpy(a).cuda() for a in v.arrays()]
        g = GridGraph(v.X, v.Y, v.Z)
        res = {}
        try:
            for mode in (0, 1, 2, 3):
                pol = Policy(learned=mode, **base)
                runs = []
                for _ in range(3):
                    g.set_tweights_device(d[0].data_ptr(), d[1].data_ptr())
                    for ax in range(3):
                        g.set_nweights_device(ax, d[2 + ax].data_ptr())
                    flow = g.max_flow(pol)
                    runs.append(g.stats())
                cuts = [hashlib.sha256(g.fill_segments(mask=1, which=k).tobytes()).hexdigest() for k in (SOURCE, SINK)]
                best = min(runs, key=lambda s: s["kernel_ms"])
                res[mode] = (flow, cuts, {k: best[k] for k in keep})
        finally:
            g.close()
        plain = res[0]
        rep = {"voxels": v.N, "schedule": repr(Policy(**base)), "plain": plain[2]}
        for mode in (1, 2, 3):
            fl, cu, st = res[mode]
            rep[f"learned{mode}"] = dict(st, mode=LEARNED_MODES[mode], speedup=plain[2]["kernel_ms"] / st["kernel_ms"],
                                         relabels_saved=plain[2]["global_relabels"] - st["global_relabels"],
                                         bit_identical=fl == plain[0] and cu == plain[1])
        out[f"workload{w}"] = rep
    return out


def generic_layered() -> dict:
    """The generic (non-grid) engine on the layered graph of the reference's
    unit_tests/graph_cut_test.cu:22-65 (100 layers of 1024 vertices, 8
    neighbours in the next layer, a 1 / 2 bottleneck in the middle layer,
    terminals of 100000 on the first and last layer; known flow 1024 * 8)."""
    import numpy as np
    from cugip_b200.graph_cut import GenericGraph
    layers, size, nbrs = 100, 1024, 8
    i = np.arange(size)
    a, b, f = [], [], []
    for layer in range(1, layers):
        w = 1 if layer == layers // 2 else 20
        for j in range(nbrs):
            a.append((layer - 1) * size + i)
            b.append(layer * size + (i + j) % size)
            f.append(np.full(size, w))
    a, b, f = np.concatenate(a), np.concatenate(b), np.concatenate(f)
    n = layers * size
    src, snk = np.zeros(n, np.int64), np.zeros(n, np.int64)
    src[:size] = 100000
    snk[-size:] = 100000
    with GenericGraph(n, a, b, f, 2 * f) as g:
        g.set_tweights(src, snk)
        runs = []
        for _ in range(4):
            flow = g.max_flow()
            runs.append(g.stats()["kernel_ms"])
        if flow != 1024 * 8:
            raise SystemExit(f"generic engine: layered flow {flow}, expected {1024 * 8}")
    return {"ms": min(runs[1:]), "vertices": n, "edges": int(a.size), "flow": flow}


def solve_kernel_name(pol) -> str:
    """The persistent solve kernel a policy launches (cgc_engine.cu launch_solve)."""
    c = pol.ctas_per_sm or 2
    if c == 2:
        return "k_solve"
    return f"k_solve{c}" + ("w" if pol.bfs_warp_min else "")


def profiled_traffic(workload: int):
    """dram bytes per k_solve launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"k_solve_workload{workload}_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


# autotune candidates: pulses, region relabels and sweep pairs per cycle, CTAs per SM, warp-per-tile BFS
# rounds and exclusive sweeps (which only the 4-CTA kernels are measured to gain from)
BATCH_CANDIDATES = [dict(local_pulses=L, region_relabels=R, sweeps_per_relabel=K, ctas_per_sm=c, bfs_warp_min=bw,
                         exclusive=ex)
                    for (L, R, K) in ((4, 2, 8), (2, 4, 4), (2, 4, 8), (4, 2, 4), (4, 4, 8), (8, 2, 8), (2, 4, 6),
                                      (4, 2, 6))
                    for c in (2, 3, 4) for bw in ((0, 8) if c > 2 else (0,)) for ex in ((0, 1) if c == 4 else (0,))]
GRID_SCHEDULES = ((4, 2, 8), (2, 4, 4), (8, 2, 8), (4, 2, 16), (2, 4, 8), (4, 4, 8), (4, 2, 6), (2, 4, 6))


def sharded_batch(dev, world, rank, steps, warmup, barrier, sha) -> dict:
    """The 96-instance batched configuration on every rank of the job: the
    instances are sharded by voxel count (shard.partition_lpt), each rank solves
    its share as one device-resident batch replayed from a CUDA graph, checks
    each of its instances (flow and both cut sets) against the oracle's golden
    answer, and the flows of all instances are gathered on every rank
    (shard.solve_sharded).  Whole-job voxels/s over the max time over ranks."""
    import torch
    import torch.distributed as dist
    from cugip_b200 import volume
    from cugip_b200.graph_cut import Batch, Policy
    from cugip_b200.shard import solve_sharded
    n = 96
    specs = [volume.preset(4, i) for i in range(n)]
    extents = [(sp.X, sp.Y, sp.Z) for sp in specs]
    gold = [golden(4, i) for i in range(n)]
    st = {}

    def check(idx, fl, outs):
        for k, i in enumerate(idx):
            if gold[i] is None:
                continue
            if fl[k] != gold[i]["flow"]:
                raise SystemExit(f"sharded batch: instance {i} flow {fl[k]} differs from the oracle's")
            if sha(outs[k][0].cpu().numpy()) != gold[i]["smin_sha256"] or \
                    sha(outs[k][1].cpu().numpy()) != gold[i]["treach_sha256"]:
                raise SystemExit(f"sharded batch: instance {i} cut sets differ from the oracle's")

    def solve_local(idx):
        vols = [volume.generate(specs[i]) for i in idx]
        ins = [[torch.from_numpy(a).to(dev) for a in v.arrays()] for v in vols]
        outs = [torch.zeros((2, v.N), dtype=torch.uint8, device=dev) for v in vols]
        B = Batch([extents[i] for i in idx])
        for k, (d, o) in enumerate(zip(ins, outs)):
            B.bind_inputs(k, d[0].data_ptr(), d[1].data_ptr(), [t.data_ptr() for t in d[2:]])
            B.bind_outputs(k, o[0].data_ptr(), o[1].data_ptr())
        best, _ = B.autotune([Policy(**c) for c in BATCH_CANDIDATES], repeats=1)
        B.graph_create(best)
        B.graph_launch()
        fl = B.wait()
        check(idx, fl, outs)
        st.update(B=B, ins=ins, outs=outs, idx=idx, best=best, voxels=sum(v.N for v in vols))
        return fl

    flows = solve_sharded(extents, solve_local)
    if any(g is not None and f != g["flow"] for f, g in zip(flows, gold)):
        raise SystemExit("sharded batch: gathered flows differ from the oracle's")
    B = st["B"]
    for _ in range(max(3, warmup)):
        B.graph_launch()
        B.wait()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        B.graph_launch()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / steps
    for o in st["outs"]:
        o.fill_(7)
    B.graph_launch()
    check(st["idx"], B.wait(), st["outs"])
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
    total = sum(x * y * z for x, y, z in extents)
    B.close()
    return {"ms": ms, "voxels_per_s": total / ms * 1e3, "voxels": total, "instances": n, "ranks": world,
            "rank0_instances": len(st["idx"]), "rank0_voxels": st["voxels"], "rank0_schedule": repr(st["best"]),
            "parity": "oracle (each rank checks its instances' flows and both cut sets)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.tmp, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            self.tmp.flush()
            for line in open(self.tmp.name):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 10:
                    continue
                if self.uuid and self.uuid not in parts[1]:
                    continue
                rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.tmp.name)
            except Exception:
                pass
        if not rows:
            return None
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(v, budget_s: float = 12.0, max_runs: int = 3):
    """Single-threaded Boykov-Kolmogorov (the oracle port of the reference's CPU
    path) on the same workload; median of up to 3 solves within the budget."""
    from oracle import oracle
    times = []
    t_start = time.time()
    while len(times) < max_runs:
        _, _, _, secs = oracle.maxflow_grid(v.X, v.Y, v.Z, v.capS, v.capT, v.n, algo=oracle.BK)
        times.append(secs)
        if time.time() - t_start > budget_s:
            break
    med = statistics.median(times)
    return {"value": v.N / med, "unit": "voxels/s", "cores": 1, "kind": "port",
            "sample": f"full {v.X}x{v.Y}x{v.Z} workload, Boykov-Kolmogorov maxflow() only, median of {len(times)}",
            "seconds": med}


_BK_CACHE = {}


def _bk_worker(workload: int) -> float:
    from cugip_b200 import volume
    from oracle import oracle
    if workload not in _BK_CACHE:
        _BK_CACHE[workload] = volume.workload(workload)
    v = _BK_CACHE[workload]
    return oracle.maxflow_grid(v.X, v.Y, v.Z, v.capS, v.capT, v.n, algo=oracle.BK)[3]


def reference_processes(voxels: int) -> int:
    """Concurrent single-threaded BK solves for the CPU arm: every core this
    process may run on, as far as host memory holds one solve per process
    (about 150 bytes per voxel at peak: volume, graph, trees and queues)."""
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = None
    by_mem = max(1, int(0.7 * avail / (150 * voxels))) if avail else cores
    return max(1, min(cores, by_mem))


def run_reference(args, rank: int, world: int):
    """CPU reference arm: the oracle's BK port on the host cores (replicas of the
    workload solved concurrently by independent processes)."""
    if rank != 0:
        return
    import multiprocessing as mp
    from cugip_b200 import volume
    v = volume.workload(args.workload)
    procs = reference_processes(v.N)
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(procs) as pool:
        for it in range(args.warmup + args.steps):
            secs = pool.map(_bk_worker, [args.workload] * procs)
            if it >= args.warmup:
                times.append(max(secs))
    ms = 1000.0 * statistics.mean(times)
    value = procs * v.N / (ms / 1000.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "voxels": v.N, "replicas": procs},
            "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": procs, "kind": "port",
                             "sample": f"{procs} concurrent single-threaded Boykov-Kolmogorov solves of the full "
                                       f"{v.X}x{v.Y}x{v.Z} workload per step (maxflow() only)"},
            "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import hashlib
    from datetime import timedelta

    import numpy as np
    import torch
    import torch.distributed as dist

    from cugip_b200 import _lib, scheduler, volume
    from cugip_b200.graph_cut import SINK, SOURCE, Batch, GridGraph, Policy

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    lib = _lib.load()
    _lib.check(lib.cgc_init(local))
    have_learned = os.path.exists(scheduler.WEIGHTS)
    if have_learned:
        scheduler.load_weights()

    def sha(t):
        return hashlib.sha256(np.ascontiguousarray(t).tobytes()).hexdigest()

    def barrier():
        if world > 1:
            dist.barrier()

    dev = torch.device("cuda", local)
    v = volume.workload(args.workload)
    N = v.N
    gold = golden(args.workload)
    d_in = [torch.from_numpy(a).to(dev) for a in v.arrays()]          # capS, capT, nx, ny, nz
    h_in = [torch.from_numpy(a).pin_memory() for a in v.arrays()]      # pinned host copies
    d_seg = torch.zeros((2, N), dtype=torch.uint8, device=dev)
    d_flow = torch.zeros(1, dtype=torch.int64, device=dev)

    # ---- production path: one-instance batch, bound device buffers, CUDA graph
    B = Batch([(v.X, v.Y, v.Z)])
    B.bind_inputs(0, d_in[0].data_ptr(), d_in[1].data_ptr(), [t.data_ptr() for t in d_in[2:]])
    B.bind_outputs(0, d_seg[0].data_ptr(), d_seg[1].data_ptr())
    cands = [Policy(local_pulses=L, region_relabels=R, sweeps_per_relabel=K, ctas_per_sm=c, learned=lr, bfs_warp_min=bw,
                    exclusive=ex)
             for (L, R, K) in GRID_SCHEDULES
             for c in (2, 3, 4) for lr in ((0, 1, 3) if have_learned else (0,)) for bw in ((0, 8) if c > 2 else (0,))
             for ex in ((0, 1) if c == 4 else (0,))]
    if args.schedule:
        L, R, K, c, lr = (int(x) for x in args.schedule.split(","))
        best, best_ms = Policy(local_pulses=L, region_relabels=R, sweeps_per_relabel=K, ctas_per_sm=c, learned=lr), None
    else:
        best, best_ms = B.autotune(cands, repeats=2)
    B.graph_create(best, d_flow.data_ptr())

    def check_outputs(flow):
        if gold is None:
            return
        if flow != gold["flow"]:
            raise SystemExit(f"flow {flow} differs from the oracle's {gold['flow']}")
        if sha(d_seg[0].cpu().numpy()) != gold["smin_sha256"] or sha(d_seg[1].cpu().numpy()) != gold["treach_sha256"]:
            raise SystemExit("cut sets differ from the oracle's")

    for _ in range(max(3, args.warmup)):
        B.graph_launch()
        check_outputs(B.wait()[0])
    d_seg.zero_()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass

    # ---- device-resident timing (graph replays)
    barrier()
    torch.cuda.synchronize()
    launches0 = lib.cgc_launch_count()
    with ClockSampler(uuid) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            B.graph_launch()
        e1.record()
        torch.cuda.synchronize()
    launches = lib.cgc_launch_count() - launches0
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    clocks = clk.summary()
    flow = B.wait()[0]
    check_outputs(flow)
    st = B.stats()

    # ---- end to end through the host API
    # Every step copies its five capacity planes from pinned host memory
    # (set_tweights / set_nweights) and its two cut sets back into pinned host
    # memory (fill_segments), inside the timed region.  Pipelined: two grids on
    # two streams, so that step i's host-to-device copies run while step i-1
    # solves (max_flow_async / wait).  Serial: one grid, one step after the other.
    g = GridGraph(v.X, v.Y, v.Z)
    hn = [t.numpy() for t in h_in]
    pipe_streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
    pipe = [GridGraph(v.X, v.Y, v.Z, stream=st.cuda_stream) for st in pipe_streams]
    h_segs = [torch.empty((2, N), dtype=torch.uint8).pin_memory() for _ in range(2)]
    hsp = [[h[0].numpy(), h[1].numpy()] for h in h_segs]
    hs = hsp[0]

    def upload(gg):
        gg.set_tweights(hn[0], hn[1])
        for ax in range(3):
            gg.set_nweights(ax, hn[2 + ax])

    def step_host():
        upload(g)
        f = g.max_flow(best)
        g.fill_segments(hs[0], 1, 0, SOURCE)
        g.fill_segments(hs[1], 1, 0, SINK)
        return f

    def run_pipelined(steps):
        flows, last = [], None
        for i in range(steps):
            gg = pipe[i % 2]
            upload(gg)
            gg.max_flow_async(best)
            if last is not None:
                k = (i - 1) % 2
                flows.append(pipe[k].wait())
                pipe[k].fill_segments(hsp[k][0], 1, 0, SOURCE)
                pipe[k].fill_segments(hsp[k][1], 1, 0, SINK)
            last = gg
        k = (steps - 1) % 2
        flows.append(pipe[k].wait())
        pipe[k].fill_segments(hsp[k][0], 1, 0, SOURCE)
        pipe[k].fill_segments(hsp[k][1], 1, 0, SINK)
        return flows

    def check_host(flows, sets):
        if gold is None:
            return
        if any(f != gold["flow"] for f in flows):
            raise SystemExit("host-API flow differs from the oracle's")
        for hsk in sets:
            if sha(hsk[0]) != gold["smin_sha256"] or sha(hsk[1]) != gold["treach_sha256"]:
                raise SystemExit("host-API cut sets differ from the oracle's")

    def timed(fn):
        barrier()
        torch.cuda.synchronize()
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record()
        out = fn()
        eb.record()
        torch.cuda.synchronize()
        barrier()
        return ea.elapsed_time(eb) / args.steps, out

    check_host(run_pipelined(2), hsp)  # warm-up of both grids
    for h in hsp:
        h[0].fill(7); h[1].fill(7)
    ms_e2e, flows_e2e = timed(lambda: run_pipelined(args.steps))
    check_host(flows_e2e, hsp if args.steps > 1 else hsp[:1])
    check_host([step_host()], [hs])
    ms_e2e_serial, f_serial = timed(lambda: [step_host() for _ in range(args.steps)])
    check_host(f_serial, [hs])

    # k_solve alone: CUDA events around its launch on the grid's stream (cgc_stats.kernel_ms)
    kms = []
    for _ in range(3):
        g.set_tweights_device(d_in[0].data_ptr(), d_in[1].data_ptr())
        for ax in range(3):
            g.set_nweights_device(ax, d_in[2 + ax].data_ptr())
        g.max_flow(best)
        kms.append(g.stats())
    solve_ms = statistics.median(s["kernel_ms"] for s in kms)

    if world > 1:
        t = torch.tensor([ms, ms_e2e, ms_e2e_serial], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_e2e_serial = float(t[0]), float(t[1]), float(t[2])

    sharded = sharded_batch(dev, world, rank, args.steps, args.warmup, barrier, sha)

    line = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        swept = statistics.median(s["tiles_swept"] for s in kms)
        relabels = statistics.median(s["global_relabels"] for s in kms)
        algo_bytes = 72.0 * 512.0 * swept + 36.0 * N * relabels
        achieved = algo_bytes / (solve_ms / 1000.0) / 1e9
        line = {
            "metric": METRIC, "value": world * N / (ms / 1000.0), "unit": "voxels/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "voxels": N,
                       "n_links": int((v.X - 1) * v.Y * v.Z + v.X * (v.Y - 1) * v.Z + v.X * v.Y * (v.Z - 1)),
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (capacities 335 MB, solver state 640 MB)",
                       "path": "device-resident batch of 1, CUDA graph replay",
                       "schedule": repr(best), "autotune_ms": best_ms},
            "e2e": {"value": world * N / (ms_e2e / 1000.0), "unit": "voxels/s",
                    "h2d_bytes_per_step": int(sum(a.nbytes for a in hn)), "d2h_bytes_per_step": int(2 * N),
                    "ms_per_step": ms_e2e,
                    "path": "GridGraph set_tweights/set_nweights from pinned host arrays, max_flow_async, wait, "
                            "fill_segments into pinned host arrays; two grids on two streams, so one step's "
                            "host-to-device copies overlap the previous step's solve",
                    "serial_value": world * N / (ms_e2e_serial / 1000.0), "serial_ms_per_step": ms_e2e_serial},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": profiled_traffic(args.workload),
                         "kernel": solve_kernel_name(best), "kernel_ms": solve_ms, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": algo_bytes},
            "solver_stats": {k: st[k] for k in ("sweeps", "global_relabels", "bfs_rounds", "tiles_swept",
                                                "tiles_relabelled", "pulses", "bfs_ms", "sweep_ms", "reach_ms",
                                                "sched_ms")},
            "flow": int(flow),
            "clocks": clocks,
            "batch96_sharded": sharded,
        }

    # ---- variants: plain vs tuned vs learned, single grid and batch
    if rank == 0 and world == 1 and not args.no_variants:
        var = {}

        def time_grid(pol, reps=5):
            ts = []
            for _ in range(reps):
                g.set_tweights_device(d_in[0].data_ptr(), d_in[1].data_ptr())
                for ax in range(3):
                    g.set_nweights_device(ax, d_in[2 + ax].data_ptr())
                e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0_.record()
                fl = g.max_flow(pol)
                g.fill_segments_device(d_seg[0].data_ptr(), 1, 0, SOURCE)
                g.fill_segments_device(d_seg[1].data_ptr(), 1, 0, SINK)
                e1_.record()
                torch.cuda.synchronize()
                ts.append(e0_.elapsed_time(e1_))
                check_outputs(fl)
            return statistics.median(ts)

        plain_ms = time_grid(Policy())
        var["grid_plain_default"] = {"ms": plain_ms, "voxels_per_s": N / plain_ms * 1e3, "schedule": repr(Policy())}
        var["grid_production"] = {"ms": ms, "voxels_per_s": N / ms * 1e3, "schedule": repr(best)}
        if have_learned:
            lp = Policy.from_options(best.options())
            lp.learned = 1
            learned_ms = time_grid(lp)
            var["grid_learned"] = {"ms": learned_ms, "voxels_per_s": N / learned_ms * 1e3, "schedule": repr(lp)}
        var["grid_speedup_production_vs_plain"] = plain_ms / ms
        # the 96-instance batched configuration
        nb = args.batch_instances
        vols = [volume.workload(4, i) for i in range(nb)]
        tot = sum(x.N for x in vols)
        dins = [[torch.from_numpy(a).to(dev) for a in x.arrays()] for x in vols]
        douts = [torch.zeros((2, x.N), dtype=torch.uint8, device=dev) for x in vols]
        gold96 = [golden(4, i) for i in range(nb)]
        have_gold96 = all(c is not None for c in gold96)

        def check_batch(fl, what):
            """every instance's flow and both bound masks against the oracle's golden answer"""
            if not have_gold96:
                if fl != seq_flows:
                    raise SystemExit(f"{what}: flows differ from the single solves")
                return
            for i, c in enumerate(gold96):
                if fl[i] != c["flow"]:
                    raise SystemExit(f"{what}: instance {i} flow {fl[i]} differs from the oracle's {c['flow']}")
                if (sha(douts[i][0].cpu().numpy()) != c["smin_sha256"]
                        or sha(douts[i][1].cpu().numpy()) != c["treach_sha256"]):
                    raise SystemExit(f"{what}: instance {i} cut sets differ from the oracle's")

        # plain: one solve per instance through the single-grid API
        seq = []
        seq_kernel_ms = []
        grids = [GridGraph(x.X, x.Y, x.Z) for x in vols]
        for rep in range(2):
            torch.cuda.synchronize()
            e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0_.record()
            for x, d, o, gg in zip(vols, dins, douts, grids):
                gg.set_tweights_device(d[0].data_ptr(), d[1].data_ptr())
                for ax in range(3):
                    gg.set_nweights_device(ax, d[2 + ax].data_ptr())
                gg.max_flow(Policy())
                gg.fill_segments_device(o[0].data_ptr(), 1, 0, SOURCE)
                gg.fill_segments_device(o[1].data_ptr(), 1, 0, SINK)
            e1_.record()
            torch.cuda.synchronize()
            seq.append(e0_.elapsed_time(e1_))
            seq_kernel_ms.append(sum(gg.stats()["kernel_ms"] for gg in grids))
        seq_flows = [gg.flow for gg in grids]
        check_batch(seq_flows, "plain sequential solves")
        for gg in grids:
            gg.close()
        seq_ms = min(seq)
        BB = Batch([(x.X, x.Y, x.Z) for x in vols])
        for i, (d, o) in enumerate(zip(dins, douts)):
            BB.bind_inputs(i, d[0].data_ptr(), d[1].data_ptr(), [t.data_ptr() for t in d[2:]])
            BB.bind_outputs(i, o[0].data_ptr(), o[1].data_ptr())
        bcands = [Policy(**c) for c in BATCH_CANDIDATES]
        bbest, _ = BB.autotune(bcands, repeats=1)

        def time_batch(pol, reps=3):
            BB.graph_create(pol)
            ts = []
            for _ in range(reps):
                for o in douts:
                    o.fill_(7)
                torch.cuda.synchronize()
                e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0_.record()
                BB.graph_launch()
                e1_.record()
                fl = BB.wait()
                ts.append(e0_.elapsed_time(e1_))
                check_batch(fl, f"batch {pol!r}")
            return statistics.median(ts)

        bat_ms = time_batch(bbest)
        var["batch96_plain_sequential"] = {"ms": seq_ms, "voxels_per_s": tot / seq_ms * 1e3, "schedule": repr(Policy()),
                                           "sum_of_kernel_ms": min(seq_kernel_ms)}
        var["batch96_parity"] = "oracle" if have_gold96 else "single solves"
        var["batch96_batched_graph"] = {"ms": bat_ms, "voxels_per_s": tot / bat_ms * 1e3, "schedule": repr(bbest)}
        if have_learned:
            modes = {}
            for mode in (1, 2, 3):
                lb = Policy.from_options(bbest.options())
                lb.learned = mode
                modes[mode] = (time_batch(lb), lb)
            mode = min(modes, key=lambda m: modes[m][0])
            lbat_ms, lb = modes[mode]
            var["batch96_learned_batched"] = {"ms": lbat_ms, "voxels_per_s": tot / lbat_ms * 1e3, "schedule": repr(lb),
                                              "ms_by_mode": {LEARNED_MODES[m]: modes[m][0] for m in modes}}
            var["batch96_speedup_learned_batched_vs_plain"] = seq_ms / lbat_ms
        var["batch96_speedup_batched_vs_plain"] = seq_ms / bat_ms
        var["batch96_voxels"] = tot
        BB.close()
        var["generic_layered"] = generic_layered()
        if have_learned:
            var["learned_config5"] = learned_report()
        line["variants"] = var

    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(v)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    g.close()
    for gg in pipe:
        gg.close()
    B.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
