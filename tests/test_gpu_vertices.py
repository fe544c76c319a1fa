"""Vertex export: every cell's vertices against the FP64 oracle.

Checks, per workload: each cell exports as many vertices as the oracle's cell
has; every vertex's planes are faces of that cell (its neighbours or box
faces); the polytope is simple (V = 2F - 4); every vertex lies within its
exported error bound of its FP64 position (the bound is rigorous), and the
position error relative to the vertex's distance from its point is at most
3e-4 * sqrt(3) (vertices looser than that are rebuilt in FP64 by the builder),
with a median below 1e-6.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _lattice(k, seed):
    rng = np.random.default_rng(seed)
    s = 1.0 / 310
    idx = np.arange(150, 150 + k, dtype=np.float64)
    g = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), -1).reshape(-1, 3)
    pts = ((g + 0.5) * s + rng.uniform(-1e-4 * s, 1e-4 * s, size=g.shape)).astype(np.float32)
    return pts, (rng.random(len(g)) * 0.1 * s * s).astype(np.float32)


def _cases():
    from paragram_b200 import workloads as W

    clouds = W.surface_clouds(num_clouds=3, seed=4, size_scale=0.05)
    return [("uniform", W.uniform(20_000, seed=3), None), ("power",) + tuple(W.power_uniform(20_000, seed=4)),
            ("clustered", W.clustered(50_000, seed=5), None), ("lattice",) + tuple(_lattice(14, 6)),
            ("surface", clouds[0], None)]


@pytest.mark.parametrize("case", range(5))
def test_vertices_match_fp64_oracle(dev, oracle, case):
    import paragram_b200 as pg
    from oracle import pg_vertex_check as V

    name, pts, w = _cases()[case]
    t = torch.from_numpy(pts).to(dev)
    tw = None if w is None else torch.from_numpy(w).to(dev)
    d, vx = pg.cell_vertices(t, tw, capacity=256)
    count = vx["count"].cpu().numpy()
    planes = vx["planes"].cpu().numpy()
    rel = vx["relative"].cpu().numpy()
    bound = vx["bound"].cpu().numpy()
    c = oracle.cells(pts, w)
    assert np.array_equal(count, c.nverts), f"{name}: vertex counts differ from the oracle"
    assert count.max() <= 256
    st = d.status.cpu().numpy()
    assert ((count == 0) == (st == 3)).all()
    rows = [set(c.rows[c.row_offsets[i]:c.row_offsets[i + 1]].tolist()) for i in range(len(pts))]
    for i in range(len(pts)):
        k = count[i]
        if k == 0:
            continue
        pl = planes[i, :k]
        faces = set(pl.ravel().tolist())
        assert {f for f in faces if f >= 0} == rows[i], f"{name}: cell {i} planes differ from its row"
        assert k == 2 * len(faces) - 4, f"{name}: cell {i} is not a simple polytope"
    lo, hi = oracle.box(pts)
    err = V.vertex_errors(pts, w, lo, hi, count, rel, bound, planes)
    print(name, err)
    assert err["over_bound"] == 0
    assert err["max_rel"] <= 3e-4 * np.sqrt(3.0)
    assert err["median_rel"] <= 1e-6
