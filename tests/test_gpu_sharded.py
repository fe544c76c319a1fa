"""One diagram built by several ranks (pg_build_range / pg_range_pack / pg_range_unpack /
pg_range_finish), the ranks run one after another on one GPU: every rank's assembled Diagram
equals the single-GPU build (and the oracle), including cells of the deferred tiers and ranges
with no cell."""

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


def _same(a, b):
    return torch.equal(a.adjacency, b.adjacency) and torch.equal(a.offsets, b.offsets) and \
        torch.equal(a.status, b.status)


@pytest.mark.parametrize("parts", [2, 3, 4])
def test_sharded_equals_single(dev, parts):
    import paragram_b200 as pg
    from paragram_b200 import sharded
    from paragram_b200 import workloads as W

    cases = [(W.clustered(100_000, seed=71), None), W.power_uniform(50_000, seed=72),
             (W.surface_cloud(40_000, np.random.default_rng(73)), None)]
    for pts, w in cases:
        t = torch.from_numpy(pts).to(dev)
        tw = None if w is None else torch.from_numpy(w).to(dev)
        ref = pg.voronoi_diagram(t) if tw is None else pg.power_diagram(t, tw)
        for d in sharded.build_shards(t, tw, parts=parts):
            assert _same(d, ref), (len(pts), parts)


def test_sharded_against_oracle_and_tiny(dev, oracle):
    from paragram_b200 import sharded
    from paragram_b200 import workloads as W

    pts = W.surface_cloud(20_000, np.random.default_rng(74))
    d = sharded.build_shards(torch.from_numpy(pts).to(dev), parts=3)[1]
    oa, oo, os_ = oracle.diagram(pts)
    assert np.array_equal(d.adjacency.cpu().numpy(), oa) and np.array_equal(d.offsets.cpu().numpy(), oo)
    assert np.array_equal(d.status.cpu().numpy(), os_)
    # more ranks than points: some ranges hold no cell
    tiny = np.random.default_rng(75).random((3, 3)).astype(np.float32)
    oa, oo, os_ = oracle.diagram(tiny)
    for d in sharded.build_shards(torch.from_numpy(tiny).to(dev), parts=5):
        assert np.array_equal(d.adjacency.cpu().numpy(), oa) and np.array_equal(d.status.cpu().numpy(), os_)


def test_range_calls_reject_bad_arguments(dev):
    from paragram_b200 import _lib

    lib = _lib.load()
    need = ctypes.c_int64(0)
    assert lib.pg_range_pack(100, None, None, 0, 10, None, 0, ctypes.byref(need), None) == -1
    ws = torch.empty(256, dtype=torch.uint8, device=dev)
    st = torch.empty(100, dtype=torch.int32, device=dev)
    assert lib.pg_range_pack(100, ws.data_ptr(), st.data_ptr(), 20, 10, None, 0, ctypes.byref(need), None) == -1
    assert lib.pg_range_unpack(100, ws.data_ptr(), st.data_ptr(), ws.data_ptr(), 10, 5, None) == -1


def test_sharded_api_single_process(dev):
    """Without a process group the sharded calls build the whole range on this GPU."""
    import paragram_b200 as pg
    from paragram_b200 import sharded
    from paragram_b200 import workloads as W

    pts, w = W.power_uniform(30_000, seed=76)
    t, tw = torch.from_numpy(pts).to(dev), torch.from_numpy(w).to(dev)
    assert _same(sharded.power_diagram(t, tw), pg.power_diagram(t, tw))
    assert _same(sharded.voronoi_diagram(t), pg.voronoi_diagram(t))
