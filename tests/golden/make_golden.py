"""Regenerates tests/golden/golden.json: for each synthetic workload the
SHA-256 of its int32 capacity volumes and the oracle's exact answer (flow,
SHA-256 of the minimal source set and of the sink-reachable set), after the
two oracle algorithms (Boykov-Kolmogorov and Dinic) agreed bit for bit.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cugip_b200 import volume  # noqa: E402
from oracle import oracle  # noqa: E402

# every instance of the 96-instance batch is pinned, not a sample of it
CASES = [(1, 0), (5, 0)] + [(4, i) for i in range(96)] + [(2, 0), (3, 0)]
DINIC_MAX_N = 3_000_000  # Dinic is cross-checked where it finishes in seconds


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def case(w, i):
    v = volume.workload(w, i)
    flow, smin, treach, secs = oracle.maxflow_grid(v.X, v.Y, v.Z, v.capS, v.capT, v.n, algo=oracle.BK)
    entry = {"workload": w, "index": i, "dims": [v.X, v.Y, v.Z], "volume_sha256": sha(*v.arrays()),
             "flow": flow, "smin_sha256": sha(smin), "treach_sha256": sha(treach),
             "smin_count": int(smin.sum()), "treach_count": int(treach.sum()), "bk_seconds": round(secs, 3)}
    if v.N <= DINIC_MAX_N:
        f2, s2, t2, _ = oracle.maxflow_grid(v.X, v.Y, v.Z, v.capS, v.capT, v.n, algo=oracle.DINIC)
        assert f2 == flow and np.array_equal(s2, smin) and np.array_equal(t2, treach), (w, i)
        entry["dinic_agrees"] = True
    assert oracle.cut_capacity_grid(v.X, v.Y, v.Z, v.capS, v.capT, v.n, None, smin) == flow
    return entry


def main():
    out = {"generator": "cgc_volume_preset/cgc_volume_generate", "cases": []}
    for w, i in CASES:
        e = case(w, i)
        print(e, flush=True)
        out["cases"].append(e)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
