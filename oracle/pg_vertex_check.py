"""FP64 reference positions of exported cell vertices (test infrastructure).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``; never by the product.

A vertex of a cell is the intersection of three planes. In coordinates
relative to the cell's point s (the frame the builder and the oracle clip in,
``pg_oracle.cpp``'s Plane), the bisector of s and q is ``a . x = beta / 2``
with ``a = q - s`` and ``beta = |q - s|^2 - (w_q - w_s)`` (the reference's
CCComputeBisectorPlane, faster_convex_cell.cuh:287-294, up to its
normalisation), and a face of the bounding box is ``x_axis = b - s_axis``
with the reference's FP32 box (voronoi_ultra.cu:234-238). The oracle solves
the same 3x3 systems in FP64; ``reference_vertices`` does it here for every
exported plane triple, so that each GPU vertex can be compared with its FP64
position and with the error bound the builder claims for it.
"""

from __future__ import annotations

from typing import Optional

import numpy as np


def reference_vertices(points, weights, box_lo, box_hi, cells, planes):
    """FP64 vertex positions relative to each vertex's cell point.

    ``cells`` int64 [V] (the cell of each vertex), ``planes`` int32 [V, 3] (point index, or
    -1 - code for a box face, code = 2 * axis + 1 on the high side). Returns float64 [V, 3].
    """
    p = np.asarray(points, dtype=np.float64)
    w = np.zeros(len(p)) if weights is None else np.asarray(weights, dtype=np.float64).reshape(-1)
    lo = np.asarray(box_lo, dtype=np.float64)
    hi = np.asarray(box_hi, dtype=np.float64)
    s = p[cells]
    A = np.zeros((len(cells), 3, 3))
    b = np.zeros((len(cells), 3))
    for e in range(3):
        ids = planes[:, e].astype(np.int64)
        bis = ids >= 0
        q = p[np.where(bis, ids, 0)]
        a = q - s
        beta = (a * a).sum(1) - (w[np.where(bis, ids, 0)] - w[cells])
        code = -1 - ids
        axis = np.where(bis, 0, code >> 1)
        face = np.where(code & 1, hi[axis], lo[axis]) - s[np.arange(len(cells)), axis]
        A[:, e, :] = np.where(bis[:, None], a, np.eye(3)[axis])
        b[:, e] = np.where(bis, 0.5 * beta, face)
    return np.linalg.solve(A, b[..., None])[..., 0]


def vertex_errors(points, weights, box_lo, box_hi, count, relative, bound, planes,
                  cells: Optional[np.ndarray] = None) -> dict:
    """Compare exported vertices with their FP64 positions.

    Returns the number of vertices, the max and median of |X - X64| / |X64| (relative to the
    vertex's distance from its cell point), the max absolute error, and how many vertices lie
    farther from their FP64 position than their exported bound (the bound is rigorous for the
    exact vertex; the FP64 solve is within ~1e-15 |X| of it).
    """
    count = np.asarray(count)
    cap = relative.shape[1]
    idx = np.arange(len(count)) if cells is None else np.asarray(cells)
    n = np.minimum(count[idx], cap)
    cell_of = np.repeat(idx, n)
    slot = np.concatenate([np.arange(k) for k in n]) if n.size else np.zeros(0, np.int64)
    rel = np.asarray(relative)[cell_of, slot].astype(np.float64)
    bnd = np.asarray(bound)[cell_of, slot].astype(np.float64)
    pl = np.asarray(planes)[cell_of, slot]
    ref = reference_vertices(points, weights, box_lo, box_hi, cell_of, pl)
    err = np.linalg.norm(rel - ref, axis=1)
    mag = np.linalg.norm(ref, axis=1)
    relerr = err / np.maximum(mag, 1e-300)
    slack = 1e-12 * mag
    return dict(vertices=int(err.size), max_rel=float(relerr.max(initial=0.0)),
                median_rel=float(np.median(relerr)) if err.size else 0.0, max_abs=float(err.max(initial=0.0)),
                over_bound=int((err > bnd + slack).sum()))
