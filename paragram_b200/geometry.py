"""Cell geometry: the volume and centroid of every cell, from the same build.

The reference clips every cell to its final polytope and keeps only the
neighbour ids (voronoi_ultra.cu:125-138, laguerre_ultra.cu:155-172). Here the
cell kernel can also integrate the final polytope before it is discarded (one
fan of tetrahedra per face, from the foot of the seed's perpendicular): the
inputs of Lloyd relaxation (centroids) and of semi-discrete optimal transport
(volumes of power cells) at the cost of the same build.
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch

from ._api import Diagram, _validate_points, _validate_weights


def cell_geometry(points: torch.Tensor, weights: Optional[torch.Tensor] = None, *, knn: int = 8,
                  leaf_size: int = -1) -> Tuple[Diagram, torch.Tensor, torch.Tensor]:
    """Build the Voronoi (``weights is None``) or power diagram and return ``(diagram, centroids, volumes)``.

    ``centroids`` is float32 [N, 3] and ``volumes`` float32 [N], both on the points' device. The
    cells are those of ``diagram`` (clipped to the reference's bounding box of the points, padded by
    1e-5). An empty power cell has volume 0 and a NaN centroid; a cell whose status is
    plane_overflow has NaN in both.
    """
    points = _validate_points(points)
    if weights is not None:
        weights = _validate_weights(weights, points.shape[0], points.device)
    from .cuda import build_with_stats

    (adjacency, offsets, status), out = build_with_stats(points, weights, knn=knn, leaf_size=leaf_size,
                                                         geometry=True)
    return Diagram(adjacency=adjacency, offsets=offsets, status=status), out["centroids"], out["volumes"]


def cell_vertices(points: torch.Tensor, weights: Optional[torch.Tensor] = None, *, capacity: int = 64,
                  knn: int = 8, leaf_size: int = -1) -> Tuple[Diagram, dict]:
    """Build the diagram and return ``(diagram, vertices)`` with every cell's vertices.

    ``vertices`` holds ``count`` (int32 [N]: vertices of each cell, 0 for an empty cell),
    ``positions`` (float32 [N, capacity, 3], absolute), ``relative`` (float32 [N, capacity, 3],
    relative to the cell's point: the precision the builder works in), ``bound`` (float32
    [N, capacity]: a rigorous bound on each vertex's distance from the exact vertex) and ``planes``
    (int32 [N, capacity, 3]: the three planes meeting at the vertex, as neighbour point indices, or
    -1 - code for a face of the bounding box, code = 2 * axis + 1 on the high side). A cell with
    more than ``capacity`` vertices keeps its first ``capacity``; unused slots hold NaN / 0.
    """
    points = _validate_points(points)
    if weights is not None:
        weights = _validate_weights(weights, points.shape[0], points.device)
    from .cuda import build_with_stats

    (adjacency, offsets, status), out = build_with_stats(points, weights, knn=knn, leaf_size=leaf_size,
                                                         vertices=capacity)
    rel = out["vertices"]
    verts = dict(count=out["vertex_count"], relative=rel, positions=rel + points[:, None, :],
                 bound=out["vertex_bound"], planes=out["vertex_planes"])
    return Diagram(adjacency=adjacency, offsets=offsets, status=status), verts


def face_areas(points: torch.Tensor, weights: Optional[torch.Tensor] = None, *, capacity: int = 64,
               knn: int = 8, leaf_size: int = -1) -> Tuple[Diagram, torch.Tensor]:
    """Build the diagram and return ``(diagram, areas)``: float32 [E], the area of the facet between
    row u and each of its neighbours, aligned with ``diagram.adjacency`` (the transport and
    finite-volume coefficients of a power diagram). Computed from the cells' exported vertices;
    NaN for a cell with more than ``capacity`` vertices (at most 256).
    """
    from . import _lib

    d, vx = cell_vertices(points, weights, capacity=capacity, knn=knn, leaf_size=leaf_size)
    points = _validate_points(points)
    n = int(points.shape[0])
    areas = torch.empty(max(d.adjacency.numel(), 1), dtype=torch.float32, device=points.device)
    if n > 0 and d.adjacency.numel() > 0:
        lib = _lib.load()
        rel = vx["relative"]
        # the library reads the exported float4 rows (x, y, z, bound)
        v4 = torch.cat([rel, vx["bound"][..., None]], dim=2).contiguous()
        with torch.cuda.device(points.device):
            rc = lib.pg_face_areas(n, int(capacity), v4.data_ptr(), vx["planes"].contiguous().data_ptr(),
                                   vx["count"].contiguous().data_ptr(), points.data_ptr(), d.offsets.data_ptr(),
                                   d.adjacency.data_ptr(), areas.data_ptr(),
                                   torch.cuda.current_stream(points.device).cuda_stream)
        if rc != 0:
            raise RuntimeError(_lib.last_error(lib))
    return d, areas[: d.adjacency.numel()]


__all__ = ["cell_geometry", "cell_vertices", "face_areas"]
