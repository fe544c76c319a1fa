"""One diagram built by several GPUs (one process per GPU, ``torch.distributed``).

Cells are independent given all points, so the work splits by cells: every
rank all-gathers the points (each rank passes its contiguous shard of the
global point order, ranks in order), builds the LBVH of all of them, builds the
cells of its own equal range of sorted slots (the LBVH's curve order, so a
range is a compact region and the ranges are balanced), packs its rows and
all-gathers the packs; every rank then assembles the full symmetric CSR and
returns the same ``Diagram`` as a single-GPU build. The exchanges are the
point all-gather (12-16 bytes per point) and the row all-gather (about 4 bytes
per directed edge plus 12 per cell); with the NCCL backend they run over
NVLink on the tensors' own devices. No reference counterpart: the reference
builds on one device.

The range build, the packing and the assembly are the library's
(``pg_build_range``, ``pg_range_pack``, ``pg_range_unpack``,
``pg_range_finish``); ``build_shards`` runs the same steps for several ranks on
one device, one after another, which is how the assembly is tested without
several GPUs.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib
from ._api import Diagram, _validate_points, _validate_weights


def _check(lib, rc):
    if rc != 0:
        raise RuntimeError(_lib.last_error(lib))


def cell_ranges(n: int, parts: int) -> list[tuple[int, int]]:
    """Equal ranges of sorted slots, one per rank."""
    return [(n * r // parts, n * (r + 1) // parts) for r in range(parts)]


class _Rank:
    """One rank's workspace and outputs."""

    def __init__(self, points: torch.Tensor, weights: Optional[torch.Tensor], begin: int, end: int,
                 leaf_size: int = -1):
        self.lib = _lib.load()
        self.n = int(points.shape[0])
        self.dev = points.device
        self.begin, self.end = begin, end
        nbytes = ctypes.c_size_t(0)
        _check(self.lib, self.lib.pg_workspace_size(self.n, ctypes.byref(nbytes)))
        self.nbytes = nbytes.value
        self.ws = torch.empty(max(self.nbytes, 1), dtype=torch.uint8, device=self.dev)
        self.status = torch.empty(max(self.n, 1), dtype=torch.int32, device=self.dev)
        self.opts = _lib.PgOptions(8, int(leaf_size), 0, 0, 0)
        self.points, self.weights = points, weights

    def _stream(self):
        return torch.cuda.current_stream(self.dev).cuda_stream

    def build(self):
        w = None if self.weights is None else self.weights.data_ptr()
        _check(self.lib, self.lib.pg_build_range(self.n, self.points.data_ptr(), w, ctypes.byref(self.opts),
                                                 self.ws.data_ptr(), self.nbytes, self.begin, self.end,
                                                 self.status.data_ptr(), self._stream()))

    def pack(self) -> torch.Tensor:
        need = ctypes.c_int64(0)
        _check(self.lib, self.lib.pg_range_pack(self.n, self.ws.data_ptr(), self.status.data_ptr(), self.begin,
                                                self.end, None, 0, ctypes.byref(need), self._stream()))
        out = torch.empty(need.value, dtype=torch.int32, device=self.dev)
        _check(self.lib, self.lib.pg_range_pack(self.n, self.ws.data_ptr(), self.status.data_ptr(), self.begin,
                                                self.end, out.data_ptr(), need.value, ctypes.byref(need),
                                                self._stream()))
        return out

    def unpack(self, pack: torch.Tensor, count: int):
        pack = pack.to(self.dev, torch.int32).contiguous()
        _check(self.lib, self.lib.pg_range_unpack(self.n, self.ws.data_ptr(), self.status.data_ptr(),
                                                  pack.data_ptr(), int(count), pack.numel(), self._stream()))

    def finish(self) -> Diagram:
        offsets = torch.empty(self.n + 1, dtype=torch.int32, device=self.dev)
        edges = ctypes.c_int64(0)
        _check(self.lib, self.lib.pg_range_finish(self.n, self.ws.data_ptr(), offsets.data_ptr(),
                                                  ctypes.byref(edges), self._stream()))
        adjacency = torch.empty(edges.value, dtype=torch.int32, device=self.dev)
        _check(self.lib, self.lib.pg_emit_adjacency(self.n, self.ws.data_ptr(), offsets.data_ptr(),
                                                    adjacency.data_ptr() if edges.value > 0 else offsets.data_ptr(),
                                                    self._stream()))
        return Diagram(adjacency=adjacency, offsets=offsets, status=self.status[: self.n])


def build_shards(points: torch.Tensor, weights: Optional[torch.Tensor] = None, parts: int = 2,
                 leaf_size: int = -1) -> list[Diagram]:
    """The diagram built as ``parts`` ranks would build it, one rank after another on the points'
    device; returns each rank's assembled Diagram (all equal to the single-GPU build)."""
    points = _validate_points(points)
    if weights is not None:
        weights = _validate_weights(weights, points.shape[0], points.device)
    n = int(points.shape[0])
    ranks = [_Rank(points, weights, b, e, leaf_size) for b, e in cell_ranges(n, parts)]
    for r in ranks:
        r.build()
    packs = [r.pack() for r in ranks]
    out = []
    for i, r in enumerate(ranks):
        for j, (p, other) in enumerate(zip(packs, ranks)):
            if j != i:
                r.unpack(p, other.end - other.begin)
        out.append(r.finish())
    return out


def exchange(local: torch.Tensor, group=None) -> list[torch.Tensor]:
    """All-gather of one 1-D tensor of any length per rank: every rank receives all of them in rank
    order (lengths first, then the tensors padded to the longest)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [local]  # one process: nothing to exchange
    world = dist.get_world_size(group)
    size = torch.tensor([local.numel()], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(size) for _ in range(world)]
    dist.all_gather(sizes, size, group=group)
    lengths = [int(s.item()) for s in sizes]
    longest = max(lengths) if lengths else 0
    padded = torch.zeros(max(longest, 1), dtype=local.dtype, device=local.device)
    padded[: local.numel()] = local
    got = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(got, padded, group=group)
    return [g[:m] for g, m in zip(got, lengths)]


def _diagram(points_local: torch.Tensor, weights_local: Optional[torch.Tensor], group, leaf_size: int) -> Diagram:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    else:
        rank, world = 0, 1
    points = torch.cat(exchange(points_local.reshape(-1), group)).reshape(-1, 3).contiguous()
    weights = None
    if weights_local is not None:
        weights = torch.cat(exchange(weights_local.reshape(-1), group)).reshape(-1, 1).contiguous()
    n = int(points.shape[0])
    ranges = cell_ranges(n, world)
    me = _Rank(points, weights, *ranges[rank], leaf_size=leaf_size)
    me.build()
    packs = exchange(me.pack(), group)
    for j, p in enumerate(packs):
        if j != rank:
            me.unpack(p, ranges[j][1] - ranges[j][0])
    return me.finish()


def voronoi_diagram(points_local: torch.Tensor, *, group=None, leaf_size: int = -1) -> Diagram:
    """Voronoi diagram of the union of every rank's points (rank r passes the r-th contiguous block
    of the global order); every rank returns the full Diagram over global point indices."""
    return _diagram(_validate_points(points_local), None, group, leaf_size)


def power_diagram(points_local: torch.Tensor, weights_local: torch.Tensor, *, group=None,
                  leaf_size: int = -1) -> Diagram:
    """Power diagram of the union of every rank's weighted points (as ``voronoi_diagram``)."""
    points_local = _validate_points(points_local)
    weights_local = _validate_weights(weights_local, points_local.shape[0], points_local.device)
    return _diagram(points_local, weights_local, group, leaf_size)


__all__ = ["build_shards", "cell_ranges", "exchange", "power_diagram", "voronoi_diagram"]
