"""Seeded synthetic point sets of the five benchmark configurations.

All generators use ``numpy.random.Generator(PCG64(seed))``, draw in float64 and
cast to float32, and return C-contiguous numpy arrays:

1. ``uniform``      N i.i.d. points in [0, 1)^3 (Voronoi).
2. ``power_uniform`` uniform points + weights U[0, 0.25 s^2], s = N^(-1/3).
3. ``clustered``    90% from 64 isotropic Gaussians (centres U[0,1)^3, sigma
                    log-uniform in [0.005, 0.1]) truncated to the cube by
                    rejection resampling, 10% uniform background, shuffled.
4. ``surface_clouds`` clouds of log-uniform size in [1e3, 5e5]; each made of
                    4-12 random planar rectangles / box surfaces, points uniform
                    by area plus Gaussian normal noise (sigma 0.002).
5. ``jittered_lattice`` m^3 lattice ((i,j,k) + 0.5) s, s = 1/m, jitter
                    U[-1e-4 s, 1e-4 s] per axis, weights U[0, 0.1 s^2].

The reference publishes no benchmark data set; these stand in for its
configurations with the stated shapes, sizes and distributions.
"""

from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def uniform(n: int, seed: int = 0) -> np.ndarray:
    return np.ascontiguousarray(_rng(seed).random((n, 3), dtype=np.float64).astype(np.float32))


def power_uniform(n: int, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    rng = _rng(seed)
    pts = rng.random((n, 3), dtype=np.float64).astype(np.float32)
    s = n ** (-1.0 / 3.0)
    w = (rng.random(n, dtype=np.float64) * 0.25 * s * s).astype(np.float32)
    return np.ascontiguousarray(pts), np.ascontiguousarray(w)


def clustered(n: int, seed: int = 0, n_clusters: int = 64, background: float = 0.1) -> np.ndarray:
    rng = _rng(seed)
    centres = rng.random((n_clusters, 3), dtype=np.float64)
    sigma = np.exp(rng.uniform(np.log(0.005), np.log(0.1), size=n_clusters))
    n_bg = int(round(n * background))
    n_cl = n - n_bg
    comp = rng.integers(0, n_clusters, size=n_cl)
    pts = centres[comp] + sigma[comp, None] * rng.standard_normal((n_cl, 3))
    bad = np.nonzero(np.any((pts < 0.0) | (pts >= 1.0), axis=1))[0]
    while bad.size:
        c = comp[bad]
        pts[bad] = centres[c] + sigma[c, None] * rng.standard_normal((bad.size, 3))
        still = np.any((pts[bad] < 0.0) | (pts[bad] >= 1.0), axis=1)
        bad = bad[still]
    allp = np.concatenate([pts, rng.random((n_bg, 3), dtype=np.float64)], axis=0)
    allp = allp[rng.permutation(n)]
    return np.ascontiguousarray(allp.astype(np.float32))


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array(
        [
            [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
            [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
            [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
        ]
    )


def surface_cloud(n: int, rng: np.random.Generator, noise: float = 0.002) -> np.ndarray:
    """One cloud: 4-12 primitives (rectangles or box surfaces), area-weighted."""
    n_prim = int(rng.integers(4, 13))
    faces = []  # (origin, u, v) with the face = origin + a u + b v, a, b in [0, 1)
    for _ in range(n_prim):
        centre = rng.uniform(0.2, 0.8, size=3)
        rot = _random_rotation(rng)
        if rng.random() < 0.5:
            w, h = rng.uniform(0.1, 0.5, size=2)
            u, v = rot[:, 0] * w, rot[:, 1] * h
            faces.append((centre - 0.5 * (u + v), u, v))
        else:
            ext = rng.uniform(0.05, 0.3, size=3)
            ax = [rot[:, k] * ext[k] for k in range(3)]
            for k in range(3):
                u, v = ax[(k + 1) % 3], ax[(k + 2) % 3]
                for sgn in (-0.5, 0.5):
                    faces.append((centre + sgn * ax[k] - 0.5 * (u + v), u, v))
    areas = np.array([np.linalg.norm(np.cross(u, v)) for _, u, v in faces])
    which = rng.choice(len(faces), size=n, p=areas / areas.sum())
    o = np.stack([faces[i][0] for i in range(len(faces))])
    U = np.stack([faces[i][1] for i in range(len(faces))])
    V = np.stack([faces[i][2] for i in range(len(faces))])
    nrm = np.cross(U, V)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    ab = rng.random((n, 2))
    pts = o[which] + ab[:, :1] * U[which] + ab[:, 1:] * V[which] + noise * rng.standard_normal((n, 1)) * nrm[which]
    return np.ascontiguousarray(pts.astype(np.float32))


def surface_clouds(num_clouds: int = 256, seed: int = 0, min_size: int = 1000, max_size: int = 500_000,
                   size_scale: float = 1.0) -> list[np.ndarray]:
    rng = _rng(seed)
    sizes = np.exp(rng.uniform(np.log(min_size), np.log(max_size), size=num_clouds))
    sizes = np.maximum((sizes * size_scale).astype(np.int64), 4)
    return [surface_cloud(int(s), rng) for s in sizes]


def jittered_lattice(m: int = 310, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    rng = _rng(seed)
    s = 1.0 / m
    idx = np.arange(m, dtype=np.float64)
    g = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), axis=-1).reshape(-1, 3)
    pts = (g + 0.5) * s + rng.uniform(-1e-4 * s, 1e-4 * s, size=g.shape)
    w = rng.random(g.shape[0], dtype=np.float64) * 0.1 * s * s
    return np.ascontiguousarray(pts.astype(np.float32)), np.ascontiguousarray(w.astype(np.float32))


#: The configuration names used by tests and bench.py.
CONFIGS = {
    "uniform_100k": "Voronoi, N=100,000 uniform in [0,1)^3",
    "power_1m": "Power diagram, N=1,000,000 uniform, weights U[0, 0.25 s^2]",
    "clustered_5m": "Voronoi, N=5,000,000: 64 Gaussian clusters (90%) + uniform background (10%)",
    "surface_256": "256 surface clouds, sizes log-uniform in [1e3, 5e5], zero weights",
    "lattice_310": "Power diagram, jittered 310^3 lattice, weights U[0, 0.1 s^2]",
}
