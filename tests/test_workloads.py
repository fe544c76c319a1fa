"""Synthetic workload generators: shapes, ranges, determinism (no GPU)."""

import numpy as np

from paragram_b200 import workloads as W


def test_uniform():
    a = W.uniform(1000, seed=1)
    assert a.dtype == np.float32 and a.shape == (1000, 3) and a.flags.c_contiguous
    assert (a >= 0).all() and (a < 1).all()
    assert np.array_equal(a, W.uniform(1000, seed=1)) and not np.array_equal(a, W.uniform(1000, seed=2))


def test_power_uniform_weights():
    p, w = W.power_uniform(8000, seed=0)
    s = 8000 ** (-1 / 3)
    assert w.shape == (8000,) and w.dtype == np.float32
    assert w.min() >= 0 and w.max() <= 0.25 * s * s + 1e-12


def test_clustered_in_cube():
    c = W.clustered(20000, seed=0)
    assert c.shape == (20000, 3) and (c >= 0).all() and (c < 1).all()
    # clustered: the densest 1% of a 20^3 grid holds far more than 1% of the points
    h, _ = np.histogramdd(c, bins=20, range=[(0, 1)] * 3)
    top = np.sort(h.ravel())[::-1][:80].sum()
    assert top > 0.1 * len(c)


def test_surface_clouds_sizes():
    clouds = W.surface_clouds(num_clouds=6, seed=3, size_scale=0.01)
    assert len(clouds) == 6
    for c in clouds:
        assert c.dtype == np.float32 and c.shape[1] == 3 and c.shape[0] >= 4


def test_jittered_lattice():
    p, w = W.jittered_lattice(8, seed=0)
    s = 1 / 8
    assert p.shape == (512, 3) and w.shape == (512,)
    g = (p / s - 0.5)
    assert np.abs(g - np.round(g)).max() <= 1e-4 + 1e-5
    assert w.max() <= 0.1 * s * s + 1e-12
