"""The C++ facade (include/cgc/graph_cut.hpp) used the way the reference's own
test uses cugip::Graph (test/graph_cut.cu:13-67)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_graph_facade.cpp")
LIBDIR = os.path.join(ROOT, "cugip_b200")


def compile_facade_test(tmp_path) -> str:
    exe = str(tmp_path / "test_graph_facade")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    SRC, "-L", LIBDIR, "-lcgc", "-lcgcvol", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_facade_compiles_against_the_c_abi(tmp_path):
    assert os.path.exists(compile_facade_test(tmp_path))


@pytest.mark.gpu
def test_facade_runs_reference_style_graph(tmp_path):
    exe = compile_facade_test(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "cpp facade ok" in out.stdout


@pytest.mark.gpu
def test_facade_exact_flow_and_reference_shaped_trace_on_512x512x128(tmp_path):
    """cugip::Graph<float> (include/cgc/cugip.hpp) on the 512x512x128 tube
    workload as an edge list: exact int64 flow and a trace object with the
    reference benchmark's hook signatures."""
    exe = compile_facade_test(tmp_path)
    out = subprocess.run([exe, "--full-size"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "full size ok" in out.stdout
