"""The bounds-checked build (libcgc_bounds.so: the engine compiled with
-DCGC_BOUNDS_CHECK, every tile, neighbour-tile and worklist index checked,
an index out of range reported as CGC_ERR_ARG instead of an access) on the
small-grid parity matrix: every solve must be exact and report no error.

It runs in a child process, because a process loads one build of the
library (the CGC_LIBRARY environment variable selects it)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BOUNDS_LIB = os.path.join(ROOT, "cugip_b200", "libcgc_bounds.so")

CHILD = r"""
import numpy as np
from cugip_b200 import _lib
from cugip_b200.graph_cut import Policy
from oracle import oracle
from tests import graphs
from tests.gpu_helpers import solve
assert _lib.LIB_PATH.endswith("libcgc_bounds.so"), _lib.LIB_PATH
policies = [None, Policy(persistent=-1), Policy(local_pulses=1, sweeps_per_relabel=1),
            Policy(ctas_per_sm=3, bfs_warp_min=1), Policy(ctas_per_sm=4, region_relabels=4, stall_sweeps=1)]
dims = [((8, 8, 8), 1), ((7, 5, 3), 2), ((16, 16, 4), 3), ((9, 1, 1), 4), ((33, 17, 9), 5), ((64, 8, 8), 6),
        ((20, 20, 20), 7), ((1, 1, 1), 8), ((40, 3, 17), 9)]
n = 0
for (X, Y, Z), seed in dims:
    capS, capT, fwd, bwd = graphs.random_grid(X, Y, Z, seed)
    f0, s0, t0, _ = oracle.maxflow_grid(X, Y, Z, capS, capT, fwd, bwd)
    for pol in policies:
        flow, smin, treach, _ = solve(X, Y, Z, capS, capT, fwd, bwd, pol)
        assert flow == f0 and np.array_equal(smin, s0) and np.array_equal(treach, t0), ((X, Y, Z), pol)
        n += 1
print("bounds ok", n)
"""


@pytest.mark.gpu
def test_bounds_checked_build_is_exact_and_finds_nothing():
    if not os.path.exists(BOUNDS_LIB):
        pytest.skip("libcgc_bounds.so is not built (cugip_b200/build.py --bounds-check)")
    env = dict(os.environ, CGC_LIBRARY=BOUNDS_LIB, PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=900)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert "bounds ok 45" in out.stdout
