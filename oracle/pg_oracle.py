"""ctypes front end of the CPU parity oracle (``pg_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg, never by the ``paragram_b200`` product.

The oracle restates the reference's construction (``paragram/_api.py:65-123``
down to ``csrc/laguerre/adjacency.cuh:78-159``) with exact predicates; see the
header of ``pg_oracle.cpp`` for the semantics and the documented differences.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpg_oracle.so")
_lib = None


class _Result(ctypes.Structure):
    _fields_ = [
        ("n_cells", ctypes.c_int64),
        ("status", ctypes.POINTER(ctypes.c_int32)),
        ("nverts", ctypes.POINTER(ctypes.c_int32)),
        ("row_offsets", ctypes.POINTER(ctypes.c_int64)),
        ("rows", ctypes.POINTER(ctypes.c_int32)),
        ("exact_calls", ctypes.c_int64),
        ("tests", ctypes.c_int64),
        ("seconds", ctypes.c_double),
        ("tree_seconds", ctypes.c_double),
        ("threads", ctypes.c_int),
    ]


def build_library(force: bool = False) -> str:
    """Compile ``libpg_oracle.so`` with the committed Makefile."""
    src = os.path.join(_HERE, "pg_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "libpg_oracle.so"], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build_library()
    lib = ctypes.CDLL(_LIB_PATH)
    f = ctypes.c_void_p
    lib.pgo_build.argtypes = [ctypes.c_int64, f, f, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                              ctypes.POINTER(_Result)]
    lib.pgo_build.restype = ctypes.c_int
    lib.pgo_free_result.argtypes = [ctypes.POINTER(_Result)]
    lib.pgo_symmetrize.argtypes = [ctypes.c_int64, f, f, f, f, ctypes.POINTER(ctypes.c_int64)]
    lib.pgo_symmetrize.restype = ctypes.c_int
    lib.pgo_side_test.argtypes = [ctypes.c_int64, f, f, ctypes.c_int64, f, f, ctypes.c_int64,
                                  ctypes.POINTER(ctypes.c_int32)]
    lib.pgo_side_test.restype = ctypes.c_int
    lib.pgo_box.argtypes = [ctypes.c_int64, f, f, f]
    _lib = lib
    return lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class OracleCells:
    """Directed per-cell output for cells [begin, end)."""

    begin: int
    status: np.ndarray        # int32 [m]
    nverts: np.ndarray        # int32 [m]
    row_offsets: np.ndarray   # int64 [m+1]
    rows: np.ndarray          # int32 [E_directed], sorted per row, original ids
    exact_calls: int
    tests: int
    seconds: float
    tree_seconds: float
    threads: int


def _prep(points, weights):
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32).reshape(-1, 3))
    w = None
    if weights is not None:
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float32).reshape(-1))
        if w.shape[0] != pts.shape[0]:
            raise ValueError("weights must have one entry per point")
    return pts, w


def cells(points, weights=None, *, mode: str = "incremental", begin: int = 0, end: Optional[int] = None,
          threads: int = 0) -> OracleCells:
    """Compute the directed rows and statuses of cells [begin, end).

    mode "incremental": kd-tree candidates + exact clipping (any N).
    mode "brute": every plane triple against every plane (N up to ~60).
    """
    lib = _load()
    pts, w = _prep(points, weights)
    n = pts.shape[0]
    end = n if end is None else end
    res = _Result()
    rc = lib.pgo_build(n, _ptr(pts), _ptr(w), 0 if mode == "incremental" else 1, begin, end, threads,
                       ctypes.byref(res))
    if rc != 0:
        raise ValueError(f"oracle rejected its arguments (rc={rc})")
    try:
        m = res.n_cells
        status = np.ctypeslib.as_array(res.status, shape=(max(m, 1),))[:m].copy()
        nverts = np.ctypeslib.as_array(res.nverts, shape=(max(m, 1),))[:m].copy()
        offs = np.ctypeslib.as_array(res.row_offsets, shape=(m + 1,)).copy()
        tot = int(offs[-1])
        rows = np.ctypeslib.as_array(res.rows, shape=(max(tot, 1),))[:tot].copy()
        return OracleCells(begin, status, nverts, offs, rows, int(res.exact_calls), int(res.tests),
                           float(res.seconds), float(res.tree_seconds), int(res.threads))
    finally:
        lib.pgo_free_result(ctypes.byref(res))


def symmetrize(n: int, offsets: np.ndarray, rows: np.ndarray):
    """Reference symmetrisation (adjacency.cuh:78-159) with sorted rows.

    Returns (adjacency int32 [E], offsets int32 [n+1]).
    """
    lib = _load()
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    adj = np.ascontiguousarray(rows, dtype=np.int32)
    out_off = np.zeros(n + 1, dtype=np.int64)
    out_adj = np.zeros(max(2 * adj.shape[0], 1), dtype=np.int32)
    out_len = ctypes.c_int64(0)
    lib.pgo_symmetrize(n, _ptr(offs), _ptr(adj), _ptr(out_off), _ptr(out_adj), ctypes.byref(out_len))
    return out_adj[: out_len.value].copy(), out_off.astype(np.int32)


def diagram(points, weights=None, *, mode: str = "incremental", threads: int = 0):
    """Full oracle diagram: (adjacency int32 [E], offsets int32 [N+1], status int32 [N])."""
    pts, w = _prep(points, weights)
    c = cells(pts, w, mode=mode, threads=threads)
    adj, off = symmetrize(pts.shape[0], c.row_offsets, c.rows)
    return adj, off, c.status


def side_test(points, weights, seed: int, kinds, ids, q: int):
    """Exact side test of one vertex against the bisector of (seed, q).

    Returns (removed: bool, used_exact: bool).
    """
    lib = _load()
    pts, w = _prep(points, weights)
    k = np.ascontiguousarray(kinds, dtype=np.int32)
    i = np.ascontiguousarray(ids, dtype=np.int32)
    used = ctypes.c_int32(0)
    r = lib.pgo_side_test(pts.shape[0], _ptr(pts), _ptr(w), seed, _ptr(k), _ptr(i), q, ctypes.byref(used))
    return bool(r), bool(used.value)


def box(points):
    """The reference's initial box (FP32): ((lo x,y,z), (hi x,y,z))."""
    lib = _load()
    pts, _ = _prep(points, None)
    lo = np.zeros(3, dtype=np.float32)
    hi = np.zeros(3, dtype=np.float32)
    lib.pgo_box(pts.shape[0], _ptr(pts), _ptr(lo), _ptr(hi))
    return lo, hi
