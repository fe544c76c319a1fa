"""CPU oracle of the cell geometry (volume and centroid of every cell).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, never by the ``paragram_b200``
product.

The reference clips each cell to its final polytope and keeps only the
neighbour ids (``paragram/csrc/laguerre/voronoi_ultra.cu:125-138``,
``laguerre_ultra.cu:155-172``), so it has no geometry output to compare with.
This oracle takes the exact facets of each cell from the parity oracle
(``pg_oracle.cells``: the cell's directed row) plus the reference's FP32 box
(``pg_oracle.box``), intersects those half-spaces in FP64 with Qhull
(``scipy.spatial.HalfspaceIntersection``, an independent implementation of the
polytope), and integrates the polytope by a fan of tetrahedra from an interior
point. It is pinned by identities any partition of the box satisfies (the
volumes sum to the box volume, the volume-weighted centroids to the box
centroid) and by a lattice whose cells are known boxes (``tests/test_geometry_oracle.py``).

Planes, relative to the seed s (power distance |x - p|^2 - w_p, as
``pg_oracle.cpp``): bisector with q: 2 (q - s).x <= |q - s|^2 - (w_q - w_s);
box face x_k = b: x_k <= b - s_k (high face) or -x_k <= s_k - b (low face).
"""

from __future__ import annotations

import numpy as np
from scipy.optimize import linprog
from scipy.spatial import ConvexHull, HalfspaceIntersection

from . import pg_oracle


def _halfspaces(pts: np.ndarray, w: np.ndarray, i: int, nbrs: np.ndarray, lo: np.ndarray, hi: np.ndarray):
    """Half-spaces [A | b] with A x + b <= 0 of cell i, in coordinates relative to its seed."""
    s = pts[i]
    d = pts[nbrs] - s
    beta = (d * d).sum(1) - (w[nbrs] - w[i])
    rows = [np.concatenate([2.0 * d, -beta[:, None]], axis=1)]
    eye = np.eye(3)
    rows.append(np.concatenate([eye, -(hi - s)[:, None]], axis=1))
    rows.append(np.concatenate([-eye, (lo - s)[:, None]], axis=1))
    return np.concatenate(rows, axis=0)


def _interior(hs: np.ndarray):
    """Chebyshev centre of {A x + b <= 0} and its radius (linear programme)."""
    a, b = hs[:, :3], hs[:, 3]
    norm = np.linalg.norm(a, axis=1)
    res = linprog(np.array([0.0, 0.0, 0.0, -1.0]), A_ub=np.concatenate([a, norm[:, None]], axis=1), b_ub=-b,
                  bounds=[(None, None)] * 3 + [(0.0, None)], method="highs")
    if not res.success:
        return None, 0.0
    return res.x[:3], float(res.x[3])


def polytope(hs: np.ndarray):
    """(volume, centroid) of {A x + b <= 0}; (0, nan) when it has no interior."""
    c, r = _interior(hs)
    if c is None or r <= 0.0:
        return 0.0, np.full(3, np.nan)
    v = HalfspaceIntersection(hs, c).intersections
    hull = ConvexHull(v)
    tri = v[hull.simplices]  # (F, 3, 3)
    e = tri - c
    vol = np.abs(np.einsum("ij,ij->i", e[:, 0], np.cross(e[:, 1], e[:, 2]))) / 6.0
    cen = (tri.sum(1) + c) / 4.0
    total = vol.sum()
    return float(total), (vol[:, None] * cen).sum(0) / total


def geometry(points, weights=None, *, threads: int = 0):
    """Per point: (centroids float64 [N, 3], volumes float64 [N], status int32 [N]).

    Cells with status 0 or 2 (complete) are integrated; an empty cell (status 3) has volume 0
    and a NaN centroid; a plane_overflow cell (status 1) NaN in both.
    """
    pts32, w32 = pg_oracle._prep(points, weights)
    n = pts32.shape[0]
    c = pg_oracle.cells(pts32, w32, threads=threads)
    lo32, hi32 = pg_oracle.box(pts32)
    pts = pts32.astype(np.float64)
    w = np.zeros(n) if w32 is None else w32.astype(np.float64)
    lo, hi = lo32.astype(np.float64), hi32.astype(np.float64)
    cen = np.full((n, 3), np.nan)
    vol = np.full(n, np.nan)
    for i in range(n):
        st = int(c.status[i])
        if st == 3:
            vol[i] = 0.0
            continue
        if st not in (0, 2):
            continue
        nbrs = c.rows[c.row_offsets[i]:c.row_offsets[i + 1]]
        v, g = polytope(_halfspaces(pts, w, i, nbrs, lo, hi))
        vol[i] = v
        cen[i] = g + pts[i]
    return cen, vol, c.status.copy()


def box_volume_and_centroid(points):
    """Volume and centroid of the reference's FP32 box, in FP64."""
    lo32, hi32 = pg_oracle.box(np.asarray(points, dtype=np.float32))
    lo, hi = lo32.astype(np.float64), hi32.astype(np.float64)
    return float(np.prod(hi - lo)), (lo + hi) / 2.0
