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
        if final_over:
            # the 512-slot tier integrates its cells too: the volumes partition the box
            _, _, vol = pg.cell_geometry(torch.from_numpy(c).to(dev))
            lo, hi = oracle.box(c)
            box = float(np.prod(hi.astype(np.float64) - lo.astype(np.float64)))
            v = vol.cpu().numpy().astype(np.float64)
            assert np.isfinite(v).all() and abs(v.sum() - box) <= 1e-5 * box


def test_batch_with_learned_radius_on_lattice_blocks(dev, oracle):
    """The near-degenerate power lattice as a batch with a learned search radius (trained on
    lattice blocks of other seeds) and a captured CUDA graph: the same diagrams as the plain batch
    and as the oracle."""
    import paragram_b200 as pg
    from paragram_b200 import learned

    def block(k, lo, seed):
        rng = np.random.default_rng(seed)
        s = 1.0 / 310
        idx = np.arange(lo, lo + k, dtype=np.float64)
        g = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), -1).reshape(-1, 3)
        pts = ((g + 0.5) * s + rng.uniform(-1e-4 * s, 1e-4 * s, size=g.shape)).astype(np.float32)
        return pts, (rng.random(len(g)) * 0.1 * s * s).astype(np.float32)

    train = [learned.collect(*[torch.from_numpy(a).to(dev) for a in block(30, 10 * s, 100 + s)]) for s in range(2)]
    model = learned.train(train, epochs=3, batch=4096)
    model.calibrate(train[0], quantile=0.98)
    clouds = [block(k, 150, 7 + k) for k in (12, 20, 9)]
    tp = [torch.from_numpy(p).to(dev) for p, _ in clouds]
    tw = [torch.from_numpy(w).to(dev) for _, w in clouds]
    plain = pg.build_batch(tp, tw)
    for rep in range(2):
        out = pg.build_batch(tp, tw, graph=True, model=model)
        for (p, w), d, e in zip(clouds, out, plain):
            got = _np(d)
            assert all(np.array_equal(a, b) for a, b in zip(got, _np(e)))
            assert all(np.array_equal(a, b) for a, b in zip(got, oracle.diagram(p, w)))


def test_batch_geometry_partition(dev):
    """Cell geometry through a batched build: per cloud, the cell volumes sum to the volume of that
    cloud's own box and the volume-weighted centroids to its centre (partition identities)."""
    import paragram_b200 as pg
    from oracle import pg_oracle
    from paragram_b200 import workloads as W

    clouds = [W.uniform(3000, seed=41), W.clustered(8000, seed=42)] + W.surface_clouds(num_clouds=2, seed=43,
                                                                                         size_scale=0.01)
    tens = [torch.from_numpy(c).to(dev) for c in clouds]
    geo = torch.zeros(sum(len(c) for c in clouds), 4, dtype=torch.float32, device=dev)
    pg.build_batch(tens, geometry_out=geo)
    g = geo.cpu().numpy().astype(np.float64)
    at = 0
    for c in clouds:
        part = g[at:at + len(c)]
        at += len(c)
        lo, hi = pg_oracle.box(c)
        lo, hi = lo.astype(np.float64), hi.astype(np.float64)
        vol = float(np.prod(hi - lo))
        assert abs(part[:, 3].sum() - vol) <= 1e-5 * vol
        cen = (part[:, :3] * part[:, 3:4]).sum(0) / part[:, 3].sum()
        assert np.abs(cen - 0.5 * (lo + hi)).max() <= 1e-5 * np.abs(hi - lo).max()
