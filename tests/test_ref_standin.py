"""The project-written stand-in for the reference's absent cuBQL dependency
(oracle/cubql_standin/) builds valid trees: the reference's traversal reads
nodes[offset], nodes[offset + 1] of inner nodes and primIDs[offset .. offset +
count) of leaves (voronoi_bvh.cuh:164-246), so those must stay in range and
cover every point once. Checked on the host, no GPU needed."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STANDIN = os.path.join(ROOT, "oracle", "cubql_standin")


def test_standin_tree_invariants(tmp_path):
    if shutil.which("g++") is None or not os.path.isdir("/usr/local/cuda/include"):
        pytest.skip("needs g++ and the CUDA headers")
    exe = tmp_path / "check_tree"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{STANDIN}", "-I/usr/local/cuda/include",
                    os.path.join(STANDIN, "check_tree.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "total bad=0" in r.stdout
