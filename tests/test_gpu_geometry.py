"""GPU cell geometry (volume and centroid per cell) against the CPU geometry oracle.

The cell kernel integrates each final cell from its FP32 vertices, so the bar is a tolerance:
per cell, |dV| <= 1e-3 V and |dc| <= 1e-3 of the cell's size plus 1e-5 of its distance from the
seed (the FP32 vertices are relative to the seed), with the median relative volume
error below 1e-5. At full size the size-independent identities of a partition of the box hold:
the volumes sum to the box volume and the volume-weighted centroids to the box centroid
(relative 1e-5, FP64 sums of the FP32 outputs).
"""

import numpy as np
import pytest
import torch

from oracle import pg_geometry_oracle as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _gpu(dev, pts, w=None):
    import paragram_b200 as pg

    t = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    wt = None if w is None else torch.from_numpy(np.ascontiguousarray(w, dtype=np.float32)).to(dev)
    d, cen, vol = pg.cell_geometry(t, wt)
    torch.cuda.synchronize()
    return d.status.cpu().numpy(), cen.cpu().numpy().astype(np.float64), vol.cpu().numpy().astype(np.float64)


def _check_vs_oracle(dev, pts, w=None):
    status, cen, vol = _gpu(dev, pts, w)
    ocen, ovol, ostatus = G.geometry(pts, w)
    np.testing.assert_array_equal(status, ostatus)
    empty = status == 3
    assert np.all(vol[empty] == 0.0) and np.all(np.isnan(cen[empty]))
    ok = (status == 0) | (status == 2)
    assert np.all(np.isfinite(vol[ok])) and np.all(np.isfinite(cen[ok]))
    rel = np.abs(vol[ok] - ovol[ok]) / ovol[ok]
    assert rel.max() <= 1e-3, f"worst relative volume error {rel.max():.3g}"
    assert np.median(rel) <= 1e-5, f"median relative volume error {np.median(rel):.3g}"
    # the vertices are FP32 relative to the seed: a power cell far from its seed carries their
    # error, a few 2^-24 of the seed distance, on top of the cell-size term
    size = np.cbrt(ovol[ok])
    far = np.linalg.norm(ocen[ok] - pts[ok].astype(np.float64), axis=1)
    dc = np.abs(cen[ok] - ocen[ok]).max(1) / (1e-3 * size + 1e-5 * far)
    assert dc.max() <= 1.0, f"worst centroid error {dc.max():.3g} of the tolerance"
    return status


def _check_partition(pts, status, cen, vol):
    vbox, cbox = G.box_volume_and_centroid(pts)
    assert not np.any(status == 1)
    assert np.all(vol[status == 3] == 0.0)
    ok = status != 3
    assert np.all(vol[ok] > 0)
    np.testing.assert_allclose(vol.sum(), vbox, rtol=1e-5)
    half = np.cbrt(vbox) / 2
    np.testing.assert_allclose((vol[ok, None] * cen[ok]).sum(0) / vbox, cbox, atol=1e-5 * half)


def test_voronoi_geometry_matches_oracle(dev):
    from paragram_b200 import workloads as W

    _check_vs_oracle(dev, W.uniform(3000, seed=7))


def test_power_geometry_matches_oracle(dev):
    from paragram_b200 import workloads as W

    p, w = W.power_uniform(3000, seed=5)
    status = _check_vs_oracle(dev, p, w)
    assert np.any(status == 3)  # empty power cells are covered


def test_large_cells_geometry_matches_oracle(dev):
    """A surface cloud whose cells reach 116 vertices: the 256-slot second pass writes them."""
    from paragram_b200 import workloads as W

    p = W.surface_cloud(3000, np.random.default_rng(3))
    status = _check_vs_oracle(dev, p)
    assert np.sum(status == 2) >= 10


def test_lattice_cells_are_known_boxes(dev):
    from oracle import pg_oracle

    m = 20
    g = (-1 + (2 * np.arange(m) + 1) / m).astype(np.float32)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    status, cen, vol = _gpu(dev, pts)
    lo, hi = pg_oracle.box(pts)
    g64 = g.astype(np.float64)
    mids = (g64[1:] + g64[:-1]) / 2
    edges = [np.concatenate([[float(lo[a])], mids, [float(hi[a])]]) for a in range(3)]
    idx = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    ext = np.stack([edges[a][idx[:, a] + 1] - edges[a][idx[:, a]] for a in range(3)], 1)
    mid = np.stack([(edges[a][idx[:, a] + 1] + edges[a][idx[:, a]]) / 2 for a in range(3)], 1)
    assert np.all(status == 0)
    np.testing.assert_allclose(vol, ext.prod(1), rtol=1e-5)
    np.testing.assert_allclose(cen, mid, atol=1e-5 * (2.0 / m))


@pytest.mark.parametrize("case", ["uniform_1m", "power_1m", "clustered_500k", "surface_cloud_191"])
def test_partition_identities_full_size(dev, case):
    from paragram_b200 import workloads as W

    w = None
    if case == "uniform_1m":
        p = W.uniform(1_000_000, seed=1)
    elif case == "power_1m":
        p, w = W.power_uniform(1_000_000, seed=2)
    elif case == "clustered_500k":
        p = W.clustered(500_000, seed=3)
    else:
        p = W.surface_clouds(num_clouds=256, seed=0)[191]
    status, cen, vol = _gpu(dev, p, w)
    _check_partition(p, status, cen, vol)
