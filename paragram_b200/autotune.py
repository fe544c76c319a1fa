"""Autotuner for the performance knobs of a workload.

The knobs change speed only, never results (the diagram is exact): the BVH leaf
size (points per leaf: one candidate batch per warp is at most 32 points), the
cell kernel's register budget (2 or 3 resident blocks of 8 warps per SM), the
number of cell-pass launches (``num_chunks``; by default the chunk plan from the
free device memory, ``PARAGRAM_MEM_FRAC``, is kept) and, with a learned model,
its routing threshold (``route_degree``: cells predicted to have at least that
many neighbours go straight to the 128-slot tier). The node-queue capacities of
the cell tiers are compile-time constants of the kernels and not tuned. ``tune``
times every combination on a representative sample on the current GPU and
returns the fastest; results are cached in memory per (device name, sample
signature, knob sets).
"""

from __future__ import annotations

import itertools
from typing import Optional, Sequence

import torch

_cache: dict = {}

LEAF_SIZES = (8, 12, 16, 24, 32)
BLOCKS_PER_SM = (2, 3)


def _time(fn, reps: int) -> float:
    fn()  # warm-up
    best = float("inf")
    for _ in range(reps):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    return best


def tune(points: torch.Tensor | Sequence[torch.Tensor], weights=None, *, reps: int = 2,
         leaf_sizes: Sequence[int] = LEAF_SIZES, blocks_per_sm: Sequence[int] = BLOCKS_PER_SM,
         num_chunks: Sequence[int] = (0,), model=None, route_degrees: Sequence[float] = (0.0,),
         key: Optional[str] = None) -> dict:
    """Fastest {leaf_size, blocks_per_sm, num_chunks, route_degree} for this sample (a tensor, or a
    list of clouds for batches, which take no chunk count). With ``model`` (a
    ``paragram_b200.learned.Model``) the builds use it and the model is left with the fastest
    ``route_degree``; ``num_chunks`` 0 keeps the memory-driven chunk plan."""
    from . import batch as _batch
    from . import cuda as _cuda

    batched = isinstance(points, (list, tuple))
    dev = (points[0].device if batched else points.device)
    sig = key or (f"batch{len(points)}x{sum(int(p.shape[0]) for p in points)}" if batched
                  else f"n{int(points.shape[0])}") + ("w" if weights is not None else "")
    chunks = (0,) if batched else tuple(num_chunks)
    routes = tuple(route_degrees) if model is not None else (None,)
    ck = (torch.cuda.get_device_name(dev), sig, tuple(leaf_sizes), tuple(blocks_per_sm), chunks, routes,
          model is not None)
    if ck in _cache:
        best = dict(_cache[ck])
        if model is not None:
            model.set_route(best["route_degree"])
        return best
    trials = []
    for leaf, bps, nch, rd in itertools.product(leaf_sizes, blocks_per_sm, chunks, routes):
        if model is not None:
            model.set_route(rd)
        if batched:
            fn = lambda leaf=leaf, bps=bps: _batch.build_batch(points, weights, leaf_size=leaf,  # noqa: E731
                                                               blocks_per_sm=bps, model=model)
        else:
            w = None if weights is None else weights.reshape(-1, 1)
            blob = None if model is None else model.blob
            fn = lambda leaf=leaf, bps=bps, nch=nch, w=w, blob=blob: _cuda._run(  # noqa: E731
                points, w, 8, False, None, None, leaf, num_chunks=nch, blocks_per_sm=bps, model=blob)
        trials.append({"leaf_size": leaf, "blocks_per_sm": bps, "num_chunks": nch, "route_degree": rd,
                       "ms": _time(fn, reps)})
    best = min(trials, key=lambda t: t["ms"])
    if model is not None:
        model.set_route(best["route_degree"])
    out = dict(best, trials=trials)
    _cache[ck] = out
    return dict(out)
