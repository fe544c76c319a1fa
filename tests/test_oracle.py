"""CPU oracle: cross-checks, known answers, golden fixtures (no GPU)."""

import glob
import itertools
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _same(a, b):
    return (np.array_equal(a.status, b.status) and np.array_equal(a.row_offsets, b.row_offsets)
            and np.array_equal(a.rows, b.rows))


@pytest.mark.parametrize("n", [2, 3, 7, 25, 45])
@pytest.mark.parametrize("weighted", [False, True])
def test_incremental_matches_brute_force(oracle, n, weighted):
    rng = np.random.default_rng(100 + n)
    pts = rng.random((n, 3)).astype(np.float32)
    w = (rng.random(n) * 0.3 * n ** (-2 / 3)).astype(np.float32) if weighted else None
    assert _same(oracle.cells(pts, w, mode="incremental"), oracle.cells(pts, w, mode="brute"))


@pytest.mark.parametrize("kind", ["lattice", "lattice_w", "duplicates", "coplanar", "cospherical"])
def test_degenerate_inputs_order_independent(oracle, kind):
    """Exact ties are broken by simulation of simplicity: clipping order cannot matter."""
    rng = np.random.default_rng(7)
    w = None
    if kind.startswith("lattice"):
        pts = np.array(list(itertools.product([0.2, 0.5, 0.8], repeat=3)), dtype=np.float32)
        if kind == "lattice_w":
            w = np.full(len(pts), 0.01, np.float32)
    elif kind == "duplicates":
        p = rng.random((10, 3)).astype(np.float32)
        pts = np.concatenate([p, p, p[:3]])
    elif kind == "coplanar":
        pts = rng.random((30, 3)).astype(np.float32)
        pts[:, 1] = 0.25
    else:
        ang = rng.random((20, 2)) * np.array([np.pi, 2 * np.pi])
        pts = (0.5 + 0.3 * np.stack([np.sin(ang[:, 0]) * np.cos(ang[:, 1]), np.sin(ang[:, 0]) * np.sin(ang[:, 1]),
                                     np.cos(ang[:, 0])], 1)).astype(np.float32)
        pts = np.concatenate([pts, [[0.5, 0.5, 0.5]]]).astype(np.float32)
    inc = oracle.cells(pts, w, mode="incremental")
    assert _same(inc, oracle.cells(pts, w, mode="brute"))
    # permuting the input permutes the output when there is no tie to break
    if kind in ("coplanar",):
        perm = rng.permutation(len(pts))
        inc2 = oracle.cells(pts[perm], mode="incremental")
        assert np.array_equal(inc2.status, inc.status[perm])


def test_known_answer_two_points(oracle):
    pts = np.array([[0.3, 0.5, 0.5], [0.7, 0.5, 0.5]], np.float32)
    adj, off, st = oracle.diagram(pts)
    assert adj.tolist() == [1, 0] and off.tolist() == [0, 1, 2] and st.tolist() == [0, 0]


def test_known_answer_single_point(oracle):
    adj, off, st = oracle.diagram(np.array([[0.5, 0.5, 0.5]], np.float32))
    assert adj.size == 0 and off.tolist() == [0, 0] and st.tolist() == [0]


def test_known_answer_collinear_chain(oracle):
    xs = [0.1, 0.3, 0.6, 0.65, 0.9]
    pts = np.array([[x, 0.5, 0.5] for x in xs], np.float32)
    adj, off, st = oracle.diagram(pts)
    rows = [adj[off[i]:off[i + 1]].tolist() for i in range(len(xs))]
    assert rows == [[1], [0, 2], [1, 3], [2, 4], [3]]


def test_known_answer_dominated_power_cell(oracle):
    """w1 - w0 = 1 puts the power bisector at x = -2, outside the box: cell 0 is empty."""
    pts = np.array([[0.4, 0.5, 0.5], [0.6, 0.5, 0.5]], np.float32)
    w = np.array([0.0, 1.0], np.float32)
    adj, off, st = oracle.diagram(pts, w)
    assert st.tolist() == [3, 0] and adj.size == 0 and off.tolist() == [0, 0, 0]


def test_known_answer_box_is_reference_box(oracle):
    pts = np.array([[0.25, -1.5, 3.0], [0.75, 2.0, 3.5]], np.float32)
    lo, hi = oracle.box(pts)
    exp_lo = (pts.min(0) - np.float32(1.0)) - np.float32(1e-5)
    exp_hi = (pts.max(0) + np.float32(1.0)) + np.float32(1e-5)
    assert np.array_equal(lo, exp_lo.astype(np.float32)) and np.array_equal(hi, exp_hi.astype(np.float32))


def test_symmetrization_rule(oracle):
    """adjacency.cuh:78-159: u->v kept iff deg(v) > 0; missing v->u added."""
    # directed rows: 0:{1,2}, 1:{} (degree 0), 2:{3}, 3:{0}
    off = np.array([0, 2, 2, 3, 4], np.int64)
    rows = np.array([1, 2, 3, 0], np.int32)
    adj, o = oracle.symmetrize(4, off, rows)
    got = [adj[o[i]:o[i + 1]].tolist() for i in range(4)]
    assert got == [[2, 3], [], [0, 3], [0, 2]]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden_fixtures(oracle, path):
    f = np.load(path)
    w = f["weights"] if "weights" in f.files else None
    adj, off, st = oracle.diagram(f["points"], w)
    assert np.array_equal(adj, f["adjacency"]) and np.array_equal(off, f["offsets"]) and np.array_equal(st, f["status"])


def test_uniform_properties(oracle):
    from paragram_b200 import workloads

    pts = workloads.uniform(3000, seed=3)
    adj, off, st = oracle.diagram(pts)
    assert (st == 0).all()
    deg = np.diff(off)
    assert 14.0 < deg.mean() < 17.0  # Poisson-Voronoi mean face count ~15.5 (fewer on the hull)
    for u in range(0, 3000, 97):
        row = adj[off[u]:off[u + 1]]
        assert (np.diff(row) > 0).all() and u not in row
        for v in row:
            assert u in adj[off[v]:off[v + 1]]
