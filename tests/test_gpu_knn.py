"""k nearest neighbours on the LBVH (pg_knn) against a brute-force float32 restatement, and the
reference's kNN warm start (knn_warm_start=True) giving the same diagram."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _brute_knn(pts: np.ndarray, k: int) -> np.ndarray:
    """Each point's k nearest other points: squared distances rounded per operation in float32
    like the kernel, ties by index, -1 where fewer exist."""
    n = len(pts)
    out = np.full((n, k), -1, np.int64)
    p = pts.astype(np.float32)
    for i in range(n):
        d = p - p[i]
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        d2[i] = np.inf
        order = np.lexsort((np.arange(n), d2))
        m = min(k, n - 1)
        out[i, :m] = order[:m]
    return out


@pytest.mark.parametrize("case", ["uniform", "clustered", "duplicates", "tiny"])
def test_knn_matches_brute_force(dev, case):
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    rng = np.random.default_rng(61)
    if case == "uniform":
        pts = W.uniform(4000, seed=61)
    elif case == "clustered":
        pts = W.clustered(4000, seed=62)
    elif case == "duplicates":
        base = rng.random((600, 3)).astype(np.float32)
        pts = np.concatenate([base, base[:300], base[:50]]).astype(np.float32)
    else:
        pts = rng.random((5, 3)).astype(np.float32)
    for k in (1, 8, 32) if case != "tiny" else (8,):
        got = pg.knn(torch.from_numpy(pts).to(dev), k).cpu().numpy()
        exp = _brute_knn(pts, k)
        assert np.array_equal(got, exp), (case, k, np.argwhere(got != exp)[:5])


def test_knn_rejects_bad_arguments(dev):
    import paragram_b200 as pg

    t = torch.rand(10, 3, device=dev)
    for k in (0, 33):
        with pytest.raises(ValueError):
            pg.knn(t, k)
    assert pg.knn(torch.zeros(0, 3, device=dev), 8).shape == (0, 8)


def test_knn_warm_start_same_diagram(dev, oracle):
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    pts, w = W.power_uniform(20000, seed=63)
    t, tw = torch.from_numpy(pts).to(dev), torch.from_numpy(w).to(dev)
    base = pg.power_diagram(t, tw)
    d = pg.power_diagram(t, tw, knn_warm_start=True)
    assert torch.equal(d.adjacency, base.adjacency) and torch.equal(d.offsets, base.offsets)
    assert torch.equal(d.status, base.status)
    oa, oo, os_ = oracle.diagram(pts, w)
    assert np.array_equal(base.adjacency.cpu().numpy(), oa) and np.array_equal(base.status.cpu().numpy(), os_)
    c = W.clustered(20000, seed=64)
    tc = torch.from_numpy(c).to(dev)
    a = pg.voronoi_diagram(tc)
    b = pg.voronoi_diagram(tc, knn=8, knn_warm_start=True)
    assert torch.equal(a.adjacency, b.adjacency) and torch.equal(a.status, b.status)
