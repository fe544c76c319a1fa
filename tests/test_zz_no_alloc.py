"""pg_degrees_to_offsets_noalloc: CSR offsets computed with the library's static
scratch (no device allocation), checked against the offsets pg_build returns.

The entry point exists for callers that cannot allocate device memory when they
call it (fixed start-up memory budgets, device memory owned by another
framework's allocator, paths that cannot take cudaMalloc's implicit
synchronisation). This file is collected last so that a failure here leaves
every other test already run.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _noalloc(lib, degrees: torch.Tensor, out: torch.Tensor) -> int:
    stream = torch.cuda.current_stream(degrees.device).cuda_stream
    return lib.pg_degrees_to_offsets_noalloc(degrees.numel(), degrees.data_ptr() if degrees.numel() else None,
                                             out.data_ptr(), stream)


def test_noalloc_offsets_match_build_offsets_twice(dev):
    import paragram_b200 as pg
    from paragram_b200 import _lib, workloads

    lib = _lib.load()
    diagrams = [pg.voronoi_diagram(torch.from_numpy(workloads.uniform(300_000, seed=31)).to(dev)),
                pg.power_diagram(*[torch.from_numpy(a).to(dev) for a in workloads.power_uniform(40_000, seed=32)])]
    for d in diagrams:  # two calls in a row, each against the existing entry point's offsets
        degrees = (d.offsets[1:] - d.offsets[:-1]).contiguous()
        out = torch.full_like(d.offsets, -7)
        assert _noalloc(lib, degrees, out) == 0, _lib.last_error(lib)
        torch.cuda.synchronize(dev)
        assert torch.equal(out.cpu(), d.offsets.cpu())


def test_noalloc_rejects_oversized_input(dev):
    from paragram_b200 import _lib

    lib = _lib.load()
    out = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = lib.pg_degrees_to_offsets_noalloc(1 << 26, out.data_ptr(), out.data_ptr(), None)
    assert rc == -1 and "static scan scratch" in _lib.last_error(lib)


def test_noalloc_empty(dev):
    from paragram_b200 import _lib

    lib = _lib.load()
    out = torch.full((1,), 5, dtype=torch.int32, device=dev)
    assert lib.pg_degrees_to_offsets_noalloc(0, None, out.data_ptr(), None) == 0
    torch.cuda.synchronize(dev)
    assert out.item() == 0


def test_noalloc_three_level_scan(dev):
    """More than 2048^2 rows: the scan recurses three levels inside the static scratch. Two
    calls in a row, each against torch's cumulative sum."""
    from paragram_b200 import _lib

    lib = _lib.load()
    g = torch.Generator(device=dev).manual_seed(5)
    for n in (5_000_001, 4_194_305):
        degrees = torch.randint(0, 40, (n,), device=dev, dtype=torch.int32, generator=g)
        exp = torch.zeros(n + 1, dtype=torch.int64, device=dev)
        exp[1:] = torch.cumsum(degrees.to(torch.int64), 0)
        out = torch.full((n + 1,), -7, dtype=torch.int32, device=dev)
        assert _noalloc(lib, degrees, out) == 0, _lib.last_error(lib)
        torch.cuda.synchronize(dev)
        assert torch.equal(out.to(torch.int64), exp)
