"""Facet areas (pg_face_areas, from the exported vertices), checked by identities.

* The facet between u and v is one polygon: the area of entry u->v equals that
  of v->u (relative 1e-4, plus 1e-7 of the mean facet area for thin facets:
  each side rounds the vertices relative to its own point).
* Divergence theorem for every cell that no box face bounds: its volume (from
  the cell kernel's own integration, an independent computation) equals
  (1/3) sum_f A_f h_f over its facets, h_f the signed distance from the cell's
  point to facet f's plane, (|q - s|^2 - (w_q - w_s)) / (2 |q - s|), which
  holds for any reference point (relative 1e-4).
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


def _cases():
    from paragram_b200 import workloads as W

    return [("uniform", W.uniform(20_000, seed=51), None), ("power",) + tuple(W.power_uniform(20_000, seed=52)),
            ("clustered", W.clustered(30_000, seed=53), None),
            ("surface", W.surface_clouds(num_clouds=1, seed=54, size_scale=0.05)[0], None)]


@pytest.mark.parametrize("case", range(4))
def test_face_areas_identities(dev, case):
    import paragram_b200 as pg

    name, pts, w = _cases()[case]
    t = torch.from_numpy(pts).to(dev)
    tw = None if w is None else torch.from_numpy(w).to(dev)
    d, areas = pg.face_areas(t, tw, capacity=256)
    _, vx = pg.cell_vertices(t, tw, capacity=256)
    _, _, vol = pg.cell_geometry(t, tw)
    adj, off = d.adjacency.cpu().numpy().astype(np.int64), d.offsets.cpu().numpy().astype(np.int64)
    a = areas.cpu().numpy().astype(np.float64)
    assert np.isfinite(a).all() and (a >= 0).all()
    n = len(pts)
    rows = np.repeat(np.arange(n), np.diff(off))
    # symmetry: entry u->v against v->u
    key = rows * n + adj
    order = np.argsort(key)
    rkey = adj * n + rows
    pos = np.searchsorted(key[order], rkey)
    pos = np.minimum(pos, len(order) - 1)
    found = key[order][pos] == rkey
    assert found.all()
    b = a[order][pos]
    scale = np.maximum(a, b)
    # FP32 rounding of the vertices relative to each cell's point: relative 1e-4 on ordinary facets,
    # plus an absolute floor of 1e-7 of the mean facet area for the thinnest ones
    floor = 1e-7 * a.mean()
    assert (np.abs(a - b) <= 1e-4 * scale + floor).all(), np.abs(a - b).max()
    # divergence theorem on cells bounded by bisectors only
    p = pts.astype(np.float64)
    ww = np.zeros(n) if w is None else w.astype(np.float64)
    q = p[adj] - p[rows]
    dq = np.linalg.norm(q, axis=1)
    h = ((dq * dq) - (ww[adj] - ww[rows])) / (2.0 * dq)
    div = np.bincount(rows, weights=a * h, minlength=n) / 3.0
    planes = vx["planes"].cpu().numpy()
    cnt = vx["count"].cpu().numpy()
    interior = np.array([cnt[i] > 0 and (planes[i, :cnt[i]] >= 0).all() for i in range(n)])
    v = vol.cpu().numpy().astype(np.float64)
    assert interior.sum() > (0 if name == "surface" else 0.5 * n)  # surface cells mostly reach the box
    rel = np.abs(div[interior] - v[interior]) / np.maximum(v[interior], 1e-30)
    print(name, "interior cells", int(interior.sum()), "max rel", float(rel.max()), "median", float(np.median(rel)))
    assert rel.max() <= 1e-4
