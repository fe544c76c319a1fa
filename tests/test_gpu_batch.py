"""Batched builds: one launch over many clouds equals one call per cloud."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _np(d):
    return d.adjacency.cpu().numpy(), d.offsets.cpu().numpy(), d.status.cpu().numpy()


@pytest.mark.parametrize("graph", [False, True])
def test_batch_equals_single_calls_and_oracle(dev, oracle, graph):
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    rng = np.random.default_rng(3)
    clouds = W.surface_clouds(num_clouds=5, seed=4, size_scale=0.01)
    clouds += [rng.random((1, 3)).astype(np.float32), rng.random((2, 3)).astype(np.float32),
               rng.random((17, 3)).astype(np.float32), W.uniform(3000, seed=5)]
    tens = [torch.from_numpy(c).to(dev) for c in clouds]
    for rep in range(2):  # second call replays the captured graph
        out = pg.build_batch(tens, graph=graph)
        assert len(out) == len(clouds)
        for c, d in zip(clouds, out):
            got = _np(d)
            exp = oracle.diagram(c)
            assert np.array_equal(got[1], exp[1]) and np.array_equal(got[0], exp[0]) and np.array_equal(got[2], exp[2])
            single = _np(pg.voronoi_diagram(torch.from_numpy(c).to(dev)))
            assert all(np.array_equal(a, b) for a, b in zip(got, single))


def test_batch_power(dev, oracle):
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    clouds = [W.power_uniform(n, seed=n) for n in (50, 700, 4000)]
    out = pg.build_batch([torch.from_numpy(p).to(dev) for p, _ in clouds],
                         [torch.from_numpy(w).to(dev) for _, w in clouds])
    for (p, w), d in zip(clouds, out):
        got = _np(d)
        exp = oracle.diagram(p, w)
        assert all(np.array_equal(a, b) for a, b in zip(got, exp))


def test_cells_beyond_256_vertices(dev, oracle):
    """Surface clouds have rare long cells that outgrow 256 vertex slots (the 512-slot tier):
    cloud 191 has a final cell of 292 vertices, cloud 56 one that exceeds 256 slots only while
    it is being clipped. Status vertex_overflow and complete sorted rows, as the oracle."""
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    clouds = W.surface_clouds(num_clouds=256, seed=0)
    for k, final_over in ((191, True), (56, False)):
        c = clouds[k]
        got = _np(pg.voronoi_diagram(torch.from_numpy(c).to(dev)))
        exp = oracle.diagram(c)
        assert all(np.array_equal(a, b) for a, b in zip(got, exp)), k
        assert (got[2] == 1).sum() == 0
        assert (oracle.cells(c).nverts.max() > 256) == final_over
