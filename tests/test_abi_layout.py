"""The host-side mirrors of the C ABI agree with include/cgc.h (no GPU).

* The ctypes structs of cugip_b200/_lib.py have the sizes and field offsets
  that the C compiler gives the structs of include/cgc.h, so options, stats
  and volume specs cross the boundary unchanged.
* cgc::GraphCutPolicy (include/cgc/graph_cut.hpp) fills every cgc_options
  field, and GraphCutPolicy::autotuned reads a cached choice back through
  cgc_autotune_lookup (host-only: the cache file named by CGC_AUTOTUNE_CACHE).
* Policy.from_options(policy.options()) keeps every field (Python facade).
"""
import ctypes as C
import math
import os
import subprocess

import pytest

from cugip_b200 import _lib, volume
from cugip_b200.graph_cut import Policy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "cugip_b200")

MIRRORS = [("cgc_options", _lib.Options), ("cgc_stats", _lib.Stats), ("cgc_volume_spec", volume.VolumeSpec)]


def _c_layout(tmp_path) -> dict:
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cgc.h"', '#include "cgc_volume.h"',
             "int main(void) {"]
    for cname, py in MIRRORS:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", INCLUDE, str(src), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    layout = {}
    for line in out.splitlines():
        struct, field, value = line.split()
        layout[(struct, field)] = int(value)
    return layout


def test_ctypes_mirrors_match_the_c_structs(tmp_path):
    layout = _c_layout(tmp_path)
    for cname, py in MIRRORS:
        assert C.sizeof(py) == layout[(cname, "sizeof")], cname
        for field, _ in py._fields_:
            assert getattr(py, field).offset == layout[(cname, field)], (cname, field)


def test_python_policy_round_trip_keeps_every_field():
    values = dict(local_pulses=3, sweeps_per_relabel=5, wait_limit_us=1000, max_sweeps=77, persistent=-1,
                  region_relabels=2, stall_sweeps=4, ctas_per_sm=3, learned=2, trace_cycles=6, bfs_warp_min=8,
                  exclusive=1, relabel=1)
    p = Policy(**values)
    o = p.options()
    assert o.struct_size == C.sizeof(_lib.Options)
    for k, v in values.items():
        assert getattr(o, k) == v, k
    back = Policy.from_options(o)
    for k, v in values.items():
        assert getattr(back, k) == v, k


CPP = r"""
#include <cstdio>
#include <cstdlib>
#include <cgc/graph_cut.hpp>

#define EXPECT(c) do { if (!(c)) { std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c); return 1; } } while (0)

int main() {
  cgc::GraphCutPolicy p;
  p.local_pulses = 3; p.region_relabels = 2; p.sweeps_per_relabel = 5; p.persistent = -1; p.wait_limit_us = 1000;
  p.max_sweeps = 77; p.stall_sweeps = 4; p.ctas_per_sm = 3; p.learned = 2; p.bfs_warp_min = 8; p.exclusive = 1;
  p.relabel = 1;
  const cgc_options o = p.options();
  EXPECT(o.struct_size == (int)sizeof(cgc_options));
  EXPECT(o.local_pulses == 3 && o.region_relabels == 2 && o.sweeps_per_relabel == 5 && o.persistent == -1);
  EXPECT(o.wait_limit_us == 1000 && o.max_sweeps == 77 && o.stall_sweeps == 4 && o.ctas_per_sm == 3);
  EXPECT(o.learned == 2 && o.bfs_warp_min == 8 && o.trace_cycles == 0 && o.exclusive == 1);
  EXPECT(o.relabel == 1);
  // the cache file holds one choice for a single 256^3 grid
  cgc::GraphCutPolicy t;
  EXPECT(cgc::GraphCutPolicy::autotuned(256LL * 256 * 256, 1, &t));
  EXPECT(t.local_pulses == 4 && t.region_relabels == 2 && t.sweeps_per_relabel == 8);
  EXPECT(t.ctas_per_sm == 3 && t.bfs_warp_min == 8 && t.stall_sweeps == 0 && t.learned == 0);
  // a line with the exclusive and relabel fields (128^3)
  cgc::GraphCutPolicy w;
  EXPECT(cgc::GraphCutPolicy::autotuned(128LL * 128 * 128, 1, &w));
  EXPECT(w.local_pulses == 2 && w.sweeps_per_relabel == 6 && w.ctas_per_sm == 4 && w.exclusive == 1 && w.relabel == 1);
  // no entry for another size class
  cgc::GraphCutPolicy u;
  EXPECT(!cgc::GraphCutPolicy::autotuned(64LL * 64 * 64, 1, &u));
  std::printf("policy ok\n");
  return 0;
}
"""


def test_cpp_policy_fills_every_option_and_reads_the_autotune_cache(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libcgc.so")):
        pytest.skip("libcgc.so is not built")
    src = tmp_path / "policy.cpp"
    src.write_text(CPP)
    exe = str(tmp_path / "policy")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", INCLUDE, str(src), "-L", LIBDIR,
                    "-lcgc", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    # size class of one instance: (0, floor(2 log2 N)); fields L R K ctas stall learned bfs_warp_min
    # [exclusive relabel] ms
    vb = math.floor(2 * math.log2(256 ** 3))
    vb128 = math.floor(2 * math.log2(128 ** 3))
    cache = tmp_path / "autotune.cache"
    cache.write_text(f"0 {vb} 4 2 8 3 0 0 8 7.5\n0 {vb128} 2 4 6 4 0 0 8 1 1 1.25\n")
    env = dict(os.environ, CGC_AUTOTUNE_CACHE=str(cache))
    out = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "policy ok" in out.stdout
