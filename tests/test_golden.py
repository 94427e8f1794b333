"""Golden fixtures: the synthetic volumes are regenerated bit for bit and the
oracle reproduces the committed exact answers."""
import hashlib
import json
import os

import numpy as np
import pytest

from cugip_b200 import volume
from oracle import oracle

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")))
CASES = {(c["workload"], c["index"]): c for c in GOLDEN["cases"]}


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("key", [k for k in CASES if k[0] != 3])
def test_generator_and_oracle_reproduce_golden(key):
    c = CASES[key]
    v = volume.workload(*key)
    assert [v.X, v.Y, v.Z] == c["dims"]
    assert sha(*v.arrays()) == c["volume_sha256"]
    flow, smin, treach, _ = oracle.maxflow_grid(v.X, v.Y, v.Z, v.capS, v.capT, v.n)
    assert flow == c["flow"]
    assert sha(smin) == c["smin_sha256"] and sha(treach) == c["treach_sha256"]
