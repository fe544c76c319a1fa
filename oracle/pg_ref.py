"""Loader of the reference's own CUDA extension built by ``oracle/build_ref.py``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and ``bench.py`` to compare
with and time against the reference's kernels; the paragram_b200 product
never imports it.

``oracle/_ref/paragram_ref.so`` holds the reference's pybind module
(paragram/csrc/ext.cpp) compiled from its unmodified sources, with a
project-written stand-in for its absent cuBQL dependency (BVH builder and kNN
query; ``oracle/cubql_standin/``). ``voronoi`` and ``power`` call it the way
``paragram.voronoi_diagram`` / ``paragram.power_diagram`` do
(paragram/_api.py:65-123: weights as an (N, 1) column), so the results are
the reference's (adjacency, offsets, status), with its row order; compare
rows after sorting them (``sort_rows``).
"""

from __future__ import annotations

import importlib.machinery
import importlib.util
import os
import time
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "paragram_ref.so")
_mod = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    """Import the compiled reference module (torch must be importable)."""
    global _mod
    if _mod is not None:
        return _mod
    if not available():
        raise ImportError("oracle/_ref/paragram_ref.so is missing; build it with `python oracle/build_ref.py`")
    import torch  # noqa: F401  (loads libtorch for the extension)

    loader = importlib.machinery.ExtensionFileLoader("paragram_ref", LIB_PATH)
    spec = importlib.util.spec_from_file_location("paragram_ref", LIB_PATH, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    _mod = mod
    return mod


def voronoi(points, *, knn: int = 8, debug: bool = False, leaf_size: int = -1, initial_guesses=None,
            initial_guesses_offsets=None):
    """The reference's build_voronoi_ultra on a CUDA (N, 3) float32 tensor (initial guesses: int32
    CUDA tensors, as its binding takes them, ext.cpp:21-29)."""
    return load().build_voronoi_ultra(points.contiguous(), knn=knn, debug=debug, initial_guesses=initial_guesses,
                                      initial_guesses_offsets=initial_guesses_offsets, leaf_size=leaf_size)


def power(points, weights, *, knn: int = 8, debug: bool = False, leaf_size: int = -1):
    """The reference's build_laguerre_voronoi_ultra; weights (N,) or (N, 1)."""
    w = weights.reshape(-1, 1).contiguous()
    return load().build_laguerre_voronoi_ultra(points.contiguous(), w, knn=knn, debug=debug, leaf_size=leaf_size)


def sort_rows(adjacency: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """Each CSR row sorted in place order (the reference's row order comes from atomics)."""
    adj = np.asarray(adjacency, dtype=np.int64).copy()
    off = np.asarray(offsets, dtype=np.int64)
    rows = np.repeat(np.arange(off.size - 1, dtype=np.int64), np.diff(off))
    order = np.lexsort((adj, rows))
    return adj[order].astype(np.int32)


def to_numpy(result):
    """(adjacency, offsets, status) tensors -> numpy with sorted rows."""
    adj, off, st = result
    off_np = off.cpu().numpy().astype(np.int32)
    return sort_rows(adj.cpu().numpy(), off_np), off_np, st.cpu().numpy().astype(np.int32)


def timed(fn, *args, steps: int = 3, warmup: int = 1, **kw) -> tuple[float, object]:
    """Median seconds of a synchronised call and its last result."""
    import torch

    out = None
    for _ in range(warmup):
        out = fn(*args, **kw)
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        out = fn(*args, **kw)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)), out


def phase_ms(fn, *args, **kw) -> Optional[dict]:
    """Run fn with debug=True and parse the reference's own phase timings from its stdout."""
    import re
    import sys
    import tempfile

    import torch

    torch.cuda.synchronize()
    sys.stdout.flush()
    fd = sys.stdout.fileno()
    saved = os.dup(fd)
    with tempfile.TemporaryFile(mode="w+b") as tmp:
        os.dup2(tmp.fileno(), fd)
        try:
            fn(*args, debug=True, **kw)
            torch.cuda.synchronize()
        finally:
            try:
                import ctypes

                ctypes.CDLL(None).fflush(None)
            except OSError:
                pass
            os.dup2(saved, fd)
            os.close(saved)
        tmp.seek(0)
        text = tmp.read().decode(errors="replace")
    out = {}
    for line in text.splitlines():
        m = re.match(r"\s*(.+?) time:\s*([0-9.eE+-]+)\s*ms", line)
        if m:
            out[m.group(1).strip()] = float(m.group(2))
    return out or None
