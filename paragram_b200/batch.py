"""Many independent point clouds in one build.

The reference builds one diagram per call (paragram/_api.py:65-123); building
N clouds is N calls, each with its own BVH build, kernel launches and host
synchronisations. ``build_batch`` concatenates the clouds and runs one build:
one radix sort whose keys carry the cloud id as a prefix (each cloud becomes
one BVH subtree with its own box), one persistent cell launch over all cells
of all clouds, one CSR pass and a single synchronisation for the total edge
count. With ``graph=True`` the whole device work of a batch shape is captured
once in a CUDA graph and replayed for later batches of the same shape.

Each returned ``Diagram`` equals ``voronoi_diagram`` / ``power_diagram`` of
that cloud alone (local point indices).
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from . import _lib
from ._api import Diagram

_graphs: dict = {}


def _check(lib, rc):
    if rc != 0:
        raise RuntimeError(_lib.last_error(lib))


class _Static:
    """Device buffers of one batch shape (reused by graph replays)."""

    def __init__(self, lib, dev, sizes, weighted):
        total = int(sum(sizes))
        self.total, self.nclouds = total, len(sizes)
        offs = [0]
        for s in sizes:
            offs.append(offs[-1] + int(s))
        self.cloud_off = torch.tensor(offs, dtype=torch.int32, device=dev)
        self.starts = self.cloud_off[:-1].to(torch.int64)
        self.pts = torch.empty(max(total, 1), 3, dtype=torch.float32, device=dev)
        self.w = torch.empty(max(total, 1), dtype=torch.float32, device=dev) if weighted else None
        nbytes = ctypes.c_size_t(0)
        _check(lib, lib.pg_batch_workspace_size(total, self.nclouds, ctypes.byref(nbytes)))
        self.ws = torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device=dev)
        self.nbytes = nbytes.value
        self.offsets = torch.empty(total + 1, dtype=torch.int32, device=dev)
        self.status = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
        self.graph = None

    def launch(self, lib, opts, stream, sync: bool) -> int:
        edges = ctypes.c_int64(0)
        rc = lib.pg_build_batch(self.total, self.nclouds, self.cloud_off.data_ptr(), self.pts.data_ptr(),
                                self.w.data_ptr() if self.w is not None else None, ctypes.byref(opts),
                                self.ws.data_ptr(), self.nbytes, self.offsets.data_ptr(), self.status.data_ptr(),
                                ctypes.byref(edges) if sync else None, stream)
        _check(lib, rc)
        return edges.value


def build_batch(points: Sequence[torch.Tensor], weights: Optional[Sequence[torch.Tensor]] = None, *,
                leaf_size: int = -1, graph: bool = False, blocks_per_sm: int = 0, model=None,
                geometry_out: Optional[torch.Tensor] = None, profile: bool = False) -> list[Diagram]:
    """Diagrams of independent clouds (Voronoi, or power when ``weights`` is given) in one build.

    ``model``: a trained ``paragram_b200.learned.Model`` (its search radius per point, predicted for
    every cloud in the same launch); the diagrams do not depend on it. ``geometry_out``: a float32
    [total points, 4] CUDA tensor (clouds concatenated in order) that receives each cell's
    centroid (x, y, z) and volume, as ``paragram_b200.cell_geometry`` does for one cloud.
    ``profile=True`` (not with ``graph``) records the phase times that
    ``paragram_b200.cuda.last_profile()`` returns.
    """
    if len(points) == 0:
        return []
    lib = _lib.load()
    dev = points[0].device
    for p in points:
        if not isinstance(p, torch.Tensor) or p.device != dev or p.dtype != torch.float32 or p.dim() != 2 or \
                p.shape[1] != 3:
            raise ValueError("every cloud must be a float32 (N, 3) tensor on the same CUDA device")
    if weights is not None:
        if len(weights) != len(points):
            raise ValueError("one weight tensor per cloud is required")
        for p, w in zip(points, weights):
            if w.device != dev or w.dtype != torch.float32 or w.numel() != p.shape[0]:
                raise ValueError("weights must be float32 with one entry per point, on the points' device")
    sizes = tuple(int(p.shape[0]) for p in points)
    blob = None
    if model is not None:
        blob = model.blob
        if blob.device != dev:
            raise ValueError("the model must live on the clouds' device")
    total_points = int(sum(int(p.shape[0]) for p in points))
    if geometry_out is not None:
        if not (isinstance(geometry_out, torch.Tensor) and geometry_out.device == dev and
                geometry_out.dtype == torch.float32 and geometry_out.is_contiguous() and
                tuple(geometry_out.shape) == (total_points, 4)):
            raise ValueError("geometry_out must be a contiguous float32 (total points, 4) tensor on the clouds' device")
    # a captured graph holds the model's and geometry's device addresses: they are part of the key
    key = (dev.index, tuple(int(p.shape[0]) for p in points), weights is not None, int(leaf_size),
           int(blocks_per_sm), None if blob is None else blob.data_ptr(),
           None if geometry_out is None else geometry_out.data_ptr())
    if profile and graph:
        raise ValueError("profile=True records host-side phase times and cannot be captured in a graph")
    opts = _lib.PgOptions(8, int(leaf_size), 2 if profile else 0, 0, int(blocks_per_sm))
    if blob is not None:
        opts.model = blob.data_ptr()
    if geometry_out is not None and total_points > 0:
        opts.geometry_out = geometry_out.data_ptr()
    with torch.cuda.device(dev):
        st = _graphs.get(key) if graph else None
        if st is None:
            st = _Static(lib, dev, sizes, weights is not None)
            if graph:
                _graphs[key] = st
        total = st.total
        if total > 0:
            torch.cat(list(points), out=st.pts[:total])
            if weights is not None:
                torch.cat([w.reshape(-1) for w in weights], out=st.w[:total])
        stream = torch.cuda.current_stream(dev)
        if graph and total > 0:
            if st.graph is None:
                # warm up once outside the capture (module loading, occupancy queries)
                st.launch(lib, opts, stream.cuda_stream, sync=True)
                g = torch.cuda.CUDAGraph()
                s2 = torch.cuda.Stream(dev)
                s2.wait_stream(stream)
                with torch.cuda.stream(s2):
                    with torch.cuda.graph(g, stream=s2):
                        st.launch(lib, opts, s2.cuda_stream, sync=False)
                stream.wait_stream(s2)
                st.graph = g
            st.graph.replay()
            edges = int(st.offsets[total].item())
            _check(lib, lib.pg_batch_check(st.ws.data_ptr(), total, st.nclouds, stream.cuda_stream))
        else:
            edges = st.launch(lib, opts, stream.cuda_stream, sync=True)
        adjacency = torch.empty(max(edges, 1), dtype=torch.int32, device=dev)
        if total > 0:
            _check(lib, lib.pg_emit_adjacency(total, st.ws.data_ptr(), st.offsets.data_ptr(), adjacency.data_ptr(),
                                              stream.cuda_stream))
        adjacency = adjacency[:edges]
        offsets = st.offsets.clone()
        status = st.status[:total].clone()
        # global -> local point ids, one kernel for all clouds
        starts = st.cloud_off.to(torch.int64)
        row_start = offsets[starts].to(torch.int64)
        per_cloud_edges = row_start[1:] - row_start[:-1]
        adjacency = adjacency - torch.repeat_interleave(starts[:-1].to(torch.int32), per_cloud_edges)
        out = []
        for c in range(len(sizes)):
            a, b = int(starts[c]), int(starts[c + 1])
            o = offsets[a:b + 1] - offsets[a]
            out.append(Diagram(adjacency=adjacency[int(row_start[c]):int(row_start[c + 1])], offsets=o,
                               status=status[a:b]))
        return out
