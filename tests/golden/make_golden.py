"""Generate the golden fixtures (tests/golden/*.npz) with the CPU oracle.

Each fixture holds the inputs (points, optional weights) and the oracle's
Diagram (adjacency, offsets, status). Every fixture is cross-checked at
generation time between the oracle's two independent constructions:
incremental exact clipping and brute-force vertex enumeration.

Run from the repository root:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pg_oracle  # noqa: E402


def cases():
    rng = np.random.Generator(np.random.PCG64(2024))
    cube = np.array(list(itertools.product([0.25, 0.75], repeat=3)), dtype=np.float32)
    yield "cube8", cube, None
    grid = np.array(list(itertools.product([0.1, 0.5, 0.9], repeat=3)), dtype=np.float32)
    yield "grid27", grid, None
    yield "grid27_weighted", grid, rng.random(27).astype(np.float32) * 0.02
    yield "uniform40", rng.random((40, 3)).astype(np.float32), None
    yield "power40", rng.random((40, 3)).astype(np.float32), (rng.random(40) * 0.2).astype(np.float32)
    dup = rng.random((12, 3)).astype(np.float32)
    yield "duplicates24", np.concatenate([dup, dup]), None
    line = np.stack([np.linspace(0.1, 0.9, 9), np.full(9, 0.5), np.full(9, 0.5)], axis=1).astype(np.float32)
    yield "collinear9", line, None
    plane = rng.random((30, 3)).astype(np.float32)
    plane[:, 2] = 0.5
    yield "coplanar30", plane, None
    tiny = (rng.random(3) + 1e-6 * rng.standard_normal((16, 3))).astype(np.float32)
    yield "near_coincident16", tiny, None


def main():
    for name, pts, w in cases():
        inc = pg_oracle.cells(pts, w, mode="incremental")
        bru = pg_oracle.cells(pts, w, mode="brute")
        assert np.array_equal(inc.status, bru.status), name
        assert np.array_equal(inc.row_offsets, bru.row_offsets), name
        assert np.array_equal(inc.rows, bru.rows), name
        adj, off = pg_oracle.symmetrize(pts.shape[0], inc.row_offsets, inc.rows)
        out = {"points": pts, "adjacency": adj, "offsets": off, "status": inc.status}
        if w is not None:
            out["weights"] = w
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(f"{name}: N={pts.shape[0]} E={adj.size} status={np.bincount(inc.status, minlength=6).tolist()}")


if __name__ == "__main__":
    main()
