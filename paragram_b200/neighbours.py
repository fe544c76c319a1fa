"""k nearest neighbours of every point (``pg_knn``), and the reference's kNN warm start.

The reference finds each point's 8 nearest points with cuBQL and clips the cell
by them before its traversal (pwr_bvh.cu:159-215, voronoi_ultra.cu:205-227).
This build's cell pass starts at the point's own BVH leaf instead, so the
drop-in calls accept ``knn`` and do not need it; ``knn`` here exports the query
and ``voronoi_diagram(..., knn_warm_start=True)`` reproduces the reference's
warm start through the initial-guess path (same diagram, more work).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


def knn(points: torch.Tensor, k: int = 8) -> torch.Tensor:
    """int32 [N, k]: per point, the original indices of its k nearest other points (unweighted FP32
    Euclidean distance, ties by index, -1 where the cloud has fewer points)."""
    if not (isinstance(points, torch.Tensor) and points.is_cuda and points.dtype == torch.float32
            and points.ndim == 2 and points.shape[1] == 3):
        raise ValueError("points must be a float32 (N, 3) CUDA tensor")
    if not 1 <= int(k) <= 32:
        raise ValueError("k must be in [1, 32]")
    lib = _lib.load()
    points = points.contiguous()
    n = int(points.shape[0])
    dev = points.device
    out = torch.empty(max(n, 1), int(k), dtype=torch.int32, device=dev)
    if n == 0:
        return out[:0]
    with torch.cuda.device(dev):
        nbytes = ctypes.c_size_t(0)
        if lib.pg_workspace_size(n, ctypes.byref(nbytes)) != 0:
            raise RuntimeError(_lib.last_error(lib))
        ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
        rc = lib.pg_knn(n, points.data_ptr(), int(k), ws.data_ptr(), nbytes.value, out.data_ptr(),
                        torch.cuda.current_stream(dev).cuda_stream)
        if rc != 0:
            raise RuntimeError(_lib.last_error(lib))
    return out


def knn_guesses(points: torch.Tensor, k: int = 8) -> tuple[torch.Tensor, torch.Tensor]:
    """``(initial_guesses, initial_guesses_offsets)`` holding each point's k nearest points."""
    nb = knn(points, k)
    n = nb.shape[0]
    offsets = torch.arange(0, n * int(k) + 1, int(k), dtype=torch.int32, device=points.device)
    return nb.reshape(-1).contiguous(), offsets


__all__ = ["knn", "knn_guesses"]
