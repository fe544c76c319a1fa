"""Low-level builders, mirroring ``paragram.cuda`` (paragram/cuda/__init__.py:1-12).

``build_voronoi_ultra`` and ``build_laguerre_voronoi_ultra`` take the arguments
of the reference's pybind functions (paragram/csrc/ext.cpp:10-29) and return the
tuple ``(adjacency, offsets, status)`` of CUDA int32 tensors. Argument errors
raise ``RuntimeError`` like the reference's C++ ASSERTs
(voronoi_ultra.cu:165-173, laguerre_ultra.cu:200-213). Importing this module
raises ``ImportError`` when the CUDA library is not built, like the
reference's ``paragram.cuda``.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import torch

from .. import _lib

_LIB = _lib.load()

#: Counter names returned by ``last_stats()`` (pg_stats in include/paragram_b200.h).
STAT_NAMES = ["tests", "fp64_escalations", "exact_escalations", "deferred_cells", "nodes", "leaves", "clips",
              "candidates", "cyc_cell", "cyc_warm", "cyc_nodes", "cyc_leaves", "cyc_clips", "cyc_out", "defer_slots",
              "defer_stack", "vertex64", "hint_hits", "hint_misses", "cyc_big"]
_last_stats: dict = {}
_last_diag: dict = {}
#: Names of the values returned by ``last_profile()`` (pg_last_profile in include/paragram_b200.h).
PROFILE_NAMES = ["launches", "lbvh_ms", "cells_ms", "deferred_ms", "csr_ms", "deferred_cells", "chunks",
                 "deferred_256", "deferred_512", "routed_cells"]


def _check(ok: bool, msg: str):
    if not ok:
        raise RuntimeError(msg)


def _run(points: torch.Tensor, weights: Optional[torch.Tensor], knn: int, debug: bool,
         initial_guesses: Optional[torch.Tensor], initial_guesses_offsets: Optional[torch.Tensor], leaf_size: int,
         num_chunks: int = 0, stats: bool = False, profile: bool = False, blocks_per_sm: int = 0,
         diagnostics: bool = False, model: Optional[torch.Tensor] = None,
         radius_hint: Optional[torch.Tensor] = None, features: bool = False, fp32_only: bool = False,
         geometry: bool = False, vertices: int = 0):
    n = int(points.shape[0])
    _check(points.device.type == "cuda", "points must be on CUDA device")
    _check(points.dtype == torch.float32, "points must be of type float")
    _check(points.dim() == 2 and points.shape[1] == 3, "points must have 3 dimensions")
    points = points.contiguous()
    dev = points.device
    wptr = None
    if weights is not None:
        _check(weights.device.type == "cuda", "weights must be on CUDA device")
        _check(weights.dtype == torch.float32, "weights must be of type float")
        _check(weights.dim() == 2 and weights.shape[1] == 1, "weights must have 1 dimension")
        _check(weights.shape[0] == n, "points and weights must have the same number of elements")
        weights = weights.contiguous()
        wptr = weights.data_ptr() if n > 0 else None
    gptr = optr = None
    if initial_guesses is not None and initial_guesses_offsets is not None:
        _check(initial_guesses.device.type == "cuda", "initial_guesses must be on CUDA device")
        _check(initial_guesses_offsets.device.type == "cuda", "initial_guesses_offsets must be on CUDA device")
        _check(initial_guesses_offsets.shape[0] == n + 1, "initial_guesses_offsets must have size num_points + 1")
        initial_guesses = initial_guesses.to(torch.int32).contiguous()
        initial_guesses_offsets = initial_guesses_offsets.to(torch.int32).contiguous()
        if initial_guesses.numel() == 0:
            initial_guesses = torch.zeros(1, dtype=torch.int32, device=dev)
        gptr, optr = initial_guesses.data_ptr(), initial_guesses_offsets.data_ptr()
    opts = _lib.PgOptions(int(knn), int(leaf_size), int(bool(debug)) | (2 if profile else 0), int(num_chunks),
                          int(blocks_per_sm))
    opts.predicates = 1 if fp32_only else 0
    if model is not None:
        _check(model.device == dev and model.dtype == torch.uint8 and model.is_contiguous(),
               "model must be a contiguous uint8 tensor (a packed pg_model) on the points' device")
        opts.model = model.data_ptr()
    if radius_hint is not None:
        _check(radius_hint.device == dev and radius_hint.dtype == torch.float32 and radius_hint.numel() == n,
               "radius_hint must be float32 with one entry per point, on the points' device")
        radius_hint = radius_hint.contiguous()
        opts.radius_hint = radius_hint.data_ptr() if n > 0 else None
    radius = work = feats = order = None
    if diagnostics:
        radius = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)
        work = torch.zeros(max(n, 1), 4, dtype=torch.int32, device=dev)
        opts.radius_out, opts.work_out = radius.data_ptr(), work.data_ptr()
    if features:
        feats = torch.zeros(max(n, 1), 16, dtype=torch.float32, device=dev)
        order = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
        opts.features_out, opts.order_out = feats.data_ptr(), order.data_ptr()
    geom = None
    if geometry:
        geom = torch.zeros(max(n, 1), 4, dtype=torch.float32, device=dev)
        opts.geometry_out = geom.data_ptr()
    vtx = vpl = vcnt = None
    if vertices:
        _check(int(vertices) > 0, "vertices must be a positive capacity per cell")
        cap = int(vertices)
        vtx = torch.full((max(n, 1), cap, 4), float("nan"), dtype=torch.float32, device=dev)
        vpl = torch.zeros(max(n, 1), cap, 3, dtype=torch.int32, device=dev)
        vcnt = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
        opts.vertex_cap = cap
        opts.vertices_out, opts.vertex_planes_out, opts.vertex_count_out = (vtx.data_ptr(), vpl.data_ptr(),
                                                                            vcnt.data_ptr())
    with torch.cuda.device(dev):
        nbytes = ctypes.c_size_t(0)
        rc = _LIB.pg_workspace_size(n, ctypes.byref(nbytes))
        _check(rc == 0, _lib.last_error(_LIB))
        ws = torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device=dev)
        offsets = torch.empty(n + 1, dtype=torch.int32, device=dev)
        status = torch.empty(n, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        edges = ctypes.c_int64(0)
        rc = _LIB.pg_build(n, points.data_ptr() if n > 0 else None, wptr, gptr, optr, ctypes.byref(opts),
                           ws.data_ptr(), nbytes.value, offsets.data_ptr(), status.data_ptr() if n > 0 else None,
                           ctypes.byref(edges), stream)
        _check(rc == 0, _lib.last_error(_LIB))
        adjacency = torch.empty(edges.value, dtype=torch.int32, device=dev)
        if n > 0:
            rc = _LIB.pg_emit_adjacency(n, ws.data_ptr(), offsets.data_ptr(),
                                        adjacency.data_ptr() if edges.value > 0 else offsets.data_ptr(), stream)
            _check(rc == 0, _lib.last_error(_LIB))
        if stats and n > 0:
            out = (ctypes.c_uint64 * len(STAT_NAMES))()
            rc = _LIB.pg_stats(ws.data_ptr(), n, out, len(STAT_NAMES), stream)
            _check(rc == 0, _lib.last_error(_LIB))
            _last_stats.clear()
            _last_stats.update({k: int(v) for k, v in zip(STAT_NAMES, out)})
    _last_diag.clear()
    if diagnostics:
        _last_diag.update(radius=radius[:n], work=work[:n])
    if features:
        _last_diag.update(features=feats[:n], order=order[:n])
    if geometry:
        _last_diag.update(centroids=geom[:n, :3], volumes=geom[:n, 3])
    if vertices:
        _last_diag.update(vertices=vtx[:n, :, :3], vertex_bound=vtx[:n, :, 3], vertex_planes=vpl[:n],
                          vertex_count=vcnt[:n])
    return adjacency, offsets, status


def last_profile() -> dict:
    """Profile of the last build on this thread (launch count; phase times if it ran with profiling)."""
    out = (ctypes.c_double * len(PROFILE_NAMES))()
    _LIB.pg_last_profile(out, len(PROFILE_NAMES))
    return {k: float(v) for k, v in zip(PROFILE_NAMES, out)}


def build_voronoi_ultra(points: torch.Tensor, knn: int = 8, debug: bool = False,
                        initial_guesses: Optional[torch.Tensor] = None,
                        initial_guesses_offsets: Optional[torch.Tensor] = None, leaf_size: int = -1):
    """Unweighted 3D Voronoi adjacency (reference: laguerre.h:24-29)."""
    return _run(points, None, knn, debug, initial_guesses, initial_guesses_offsets, leaf_size)


def build_laguerre_voronoi_ultra(points: torch.Tensor, weights: torch.Tensor, knn: int = 8, debug: bool = False,
                                 initial_guesses: Optional[torch.Tensor] = None,
                                 initial_guesses_offsets: Optional[torch.Tensor] = None, leaf_size: int = -1):
    """Weighted 3D power-diagram adjacency (reference: laguerre.h:13-20)."""
    return _run(points, weights, knn, debug, initial_guesses, initial_guesses_offsets, leaf_size)


def build_with_stats(points: torch.Tensor, weights: Optional[torch.Tensor] = None, *, knn: int = 8,
                     leaf_size: int = -1, num_chunks: int = 0, profile: bool = False, blocks_per_sm: int = 0,
                     initial_guesses: Optional[torch.Tensor] = None,
                     initial_guesses_offsets: Optional[torch.Tensor] = None, diagnostics: bool = False,
                     model: Optional[torch.Tensor] = None, radius_hint: Optional[torch.Tensor] = None,
                     features: bool = False, fp32_only: bool = False, geometry: bool = False,
                     vertices: int = 0):
    """Build and return ``((adjacency, offsets, status), counters)``; counters as in ``STAT_NAMES``.

    With ``diagnostics=True`` the counters also hold ``radius`` (float32 [N], the certified radius
    of each final cell) and ``work`` (int32 [N, 4]: BVH nodes visited, leaves visited, candidates
    tested, peak node-queue length). ``model`` is a packed learned-radius model (uint8 tensor);
    ``radius_hint`` (float32 [N]) gives a search radius per point instead. With ``features=True``
    the counters also hold ``features`` (float32 [N, 16], the learned model's inputs) and
    ``order`` (int32 [N], the curve order: sorted slot -> point index). ``fp32_only`` decides every
    side test by its FP32 value (no FP64 / exact escalation; the result may differ from the exact
    diagram on near-degenerate input). With ``geometry=True`` the counters also hold ``centroids``
    (float32 [N, 3]) and ``volumes`` (float32 [N]) of the cells (empty cell: volume 0, NaN centroid).
    With ``vertices=C`` (a capacity per cell) the counters also hold ``vertices`` (float32 [N, C, 3],
    each cell's vertices relative to its point), ``vertex_bound`` (float32 [N, C]: a rigorous bound
    on each vertex's distance from the exact vertex), ``vertex_planes`` (int32 [N, C, 3]: the planes
    meeting there, as neighbour point indices or -1 - code for a box face, code = 2 * axis + 1 on
    the high side) and ``vertex_count`` (int32 [N]); unused slots hold NaN / 0.
    """
    if weights is not None and weights.dim() == 1:
        weights = weights[:, None]
    res = _run(points, weights, knn, False, initial_guesses, initial_guesses_offsets, leaf_size,
               num_chunks=num_chunks, stats=True, profile=profile, blocks_per_sm=blocks_per_sm,
               diagnostics=diagnostics, model=model, radius_hint=radius_hint, features=features,
               fp32_only=fp32_only, geometry=geometry, vertices=vertices)
    out = dict(_last_stats)
    out.update(_last_diag)
    return res, out


__all__ = ["build_laguerre_voronoi_ultra", "build_voronoi_ultra", "build_with_stats", "last_profile", "STAT_NAMES",
           "PROFILE_NAMES"]
