"""Autotuner for the performance knobs of a workload.

The knobs change speed only, never results (the diagram is exact): the BVH leaf
size (points per leaf: one candidate batch per warp is at most 32 points) and
the cell kernel's register budget (2 or 3 resident blocks of 8 warps per SM).
The number of cell-pass launches is chosen from the free device memory
(``PARAGRAM_MEM_FRAC``), not timed. ``tune`` times every combination on a
representative sample on the current GPU and returns the fastest; results are
cached in memory per (device name, sample signature).
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
         key: Optional[str] = None) -> dict:
    """Fastest {leaf_size, blocks_per_sm} for this sample (a tensor, or a list of clouds for batches)."""
    from . import batch as _batch
    from . import cuda as _cuda

    batched = isinstance(points, (list, tuple))
    dev = (points[0] if batched else points).device
    sig = key or (f"batch{len(points)}x{sum(int(p.shape[0]) for p in points)}" if batched
                  else f"n{int(points.shape[0])}") + ("w" if weights is not None else "")
    ck = (torch.cuda.get_device_name(dev), sig)
    if ck in _cache:
        return dict(_cache[ck])
    trials = []
    for leaf, bps in itertools.product(leaf_sizes, blocks_per_sm):
        if batched:
            fn = lambda: _batch.build_batch(points, weights, leaf_size=leaf, blocks_per_sm=bps)  # noqa: E731
        else:
            w = None if weights is None else weights.reshape(-1, 1)
            fn = lambda: _cuda._run(points, w, 8, False, None, None, leaf, blocks_per_sm=bps)  # noqa: E731
        trials.append({"leaf_size": leaf, "blocks_per_sm": bps, "ms": _time(fn, reps)})
    best = min(trials, key=lambda t: t["ms"])
    out = dict(best, trials=trials)
    _cache[ck] = out
    return dict(out)
