"""The product's exact side test (paragram_b200/csrc/pg_exact.cuh), compiled for the
host with g++, against the oracle's independent big-integer evaluation (no GPU)."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("pgx") / "libpgx.so")
    src = os.path.join(ROOT, "tests", "native", "exact_harness.cpp")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", out, src], check=True)
    lib = ctypes.CDLL(out)
    vp = ctypes.c_void_p
    lib.pgx_side_test.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int]
    lib.pgx_side_test.restype = ctypes.c_int
    return lib


def _call(lib, oracle, pts, w, seed, planes, q, stage):
    lo, hi = oracle.box(pts)
    s4 = np.array([*pts[seed], w[seed] if w is not None else 0.0], np.float32)
    P = np.zeros((3, 4), np.float32)
    bx = np.full(3, -1, np.int32)
    oid = np.full(3, -1, np.int32)
    for i, (kind, idx) in enumerate(planes):
        if kind == 0:
            P[i, :3] = pts[idx]
            P[i, 3] = w[idx] if w is not None else 0.0
            oid[i] = idx
        else:
            P[i, 0] = hi[idx >> 1] if idx & 1 else lo[idx >> 1]
            bx[i] = idx
    c4 = np.array([*pts[q], w[q] if w is not None else 0.0], np.float32)
    return lib.pgx_side_test(s4.ctypes.data, seed, P.ctypes.data, bx.ctypes.data, oid.ctypes.data, c4.ctypes.data,
                             q, stage)


@pytest.mark.parametrize("family", ["random", "lattice", "clustered_ties", "boxes"])
def test_side_test_matches_oracle(harness, oracle, family):
    rng = np.random.default_rng({"random": 1, "lattice": 2, "clustered_ties": 3, "boxes": 4}[family])
    undecided_fp64 = 0
    for trial in range(400):
        n = 8
        if family == "random":
            pts = rng.random((n, 3)).astype(np.float32)
        elif family == "lattice":
            pts = (rng.integers(0, 4, (n, 3)) / 4).astype(np.float32)
        elif family == "clustered_ties":
            pts = (rng.random(3) + 1e-6 * rng.standard_normal((n, 3))).astype(np.float32)
        else:
            pts = rng.random((n, 3)).astype(np.float32)
        w = None if trial % 2 else (rng.random(n) * 0.01).astype(np.float32)
        planes = [(1, int(rng.integers(6))), (0, 1), (0, 2)] if family == "boxes" else [(0, 1), (0, 2), (0, 3)]
        ref, _ = oracle.side_test(pts, w, 0, [k for k, _ in planes], [i for _, i in planes], 4)
        assert _call(harness, oracle, pts, w, 0, planes, 4, 0) == int(ref)
        assert _call(harness, oracle, pts, w, 0, planes, 4, 2) == int(ref)
        r1 = _call(harness, oracle, pts, w, 0, planes, 4, 1)
        if r1 < 0:
            undecided_fp64 += 1
        else:
            assert r1 == int(ref)
    if family == "random":
        assert undecided_fp64 == 0
