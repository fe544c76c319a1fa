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


__all__ = ["cell_geometry"]
