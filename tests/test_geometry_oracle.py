"""Pins of the cell-geometry oracle (CPU): identities of a partition of the box, and a lattice
whose cells are known boxes."""

import numpy as np
import pytest

from oracle import pg_geometry_oracle as G
from oracle import pg_oracle


@pytest.mark.parametrize("weighted", [False, True])
def test_cells_partition_the_box(weighted):
    rng = np.random.default_rng(11 + weighted)
    p = rng.uniform(-1, 1, (400, 3)).astype(np.float32)
    w = rng.uniform(0, 0.05, 400).astype(np.float32) if weighted else None
    cen, vol, status = G.geometry(p, w)
    vbox, cbox = G.box_volume_and_centroid(p)
    assert np.all(status != 1)
    assert np.all(vol[status == 3] == 0.0)
    ok = status != 3
    assert np.all(vol[ok] > 0)
    np.testing.assert_allclose(vol.sum(), vbox, rtol=1e-12)
    np.testing.assert_allclose((vol[ok, None] * cen[ok]).sum(0) / vbox, cbox, atol=1e-12)


def test_lattice_cells_are_known_boxes():
    m = 5
    g = (-1 + (2 * np.arange(m) + 1) / m).astype(np.float32)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    cen, vol, status = G.geometry(pts)
    lo, hi = pg_oracle.box(pts)
    # per axis: the slab of lattice coordinate k runs between the midpoints (box faces at the ends)
    g64 = g.astype(np.float64)
    mids = (g64[1:] + g64[:-1]) / 2
    edges = [np.concatenate([[float(lo[a])], mids, [float(hi[a])]]) for a in range(3)]
    idx = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    ext = np.stack([edges[a][idx[:, a] + 1] - edges[a][idx[:, a]] for a in range(3)], 1)
    mid = np.stack([(edges[a][idx[:, a] + 1] + edges[a][idx[:, a]]) / 2 for a in range(3)], 1)
    np.testing.assert_allclose(vol, ext.prod(1), rtol=1e-9)
    np.testing.assert_allclose(cen, mid, atol=1e-9)
