"""GPU parity: the CUDA builder (through the C ABI) against the CPU oracle.

Bar: bit-identical sorted rows, offsets and statuses. Sizes are chosen so the
oracle finishes in seconds; the full-size configurations are covered by
size-independent properties (symmetry, sorted rows, no self loops, offsets).
"""

import glob
import itertools
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _gpu(dev, pts, w=None, **kw):
    import paragram_b200 as pg

    t = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    if w is None:
        d = pg.voronoi_diagram(t, **kw)
    else:
        d = pg.power_diagram(t, torch.from_numpy(np.ascontiguousarray(w)).to(dev), **kw)
    torch.cuda.synchronize()
    return d.adjacency.cpu().numpy(), d.offsets.cpu().numpy(), d.status.cpu().numpy()


def _assert_same(got, exp, tag=""):
    adj, off, st = got
    eadj, eoff, est = exp
    assert off.dtype == np.int32 and adj.dtype == np.int32 and st.dtype == np.int32
    if not (np.array_equal(off, eoff) and np.array_equal(adj, eadj) and np.array_equal(st, est)):
        bad = [i for i in range(len(st)) if st[i] != est[i] or not np.array_equal(
            adj[off[i]:off[i + 1]] if i + 1 < len(off) else [], eadj[eoff[i]:eoff[i + 1]])]
        raise AssertionError(f"{tag}: {len(bad)} cells differ, first {bad[:5]}")


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 64, 1000, 20000])
def test_uniform_voronoi(dev, oracle, n):
    from paragram_b200 import workloads as W

    pts = W.uniform(n, seed=n)
    _assert_same(_gpu(dev, pts), oracle.diagram(pts), f"uniform{n}")


def test_uniform_100k(dev, oracle):
    from paragram_b200 import workloads as W

    pts = W.uniform(100_000, seed=0)
    _assert_same(_gpu(dev, pts), oracle.diagram(pts), "uniform100k")


@pytest.mark.parametrize("n", [1000, 50_000])
def test_power_uniform_with_empty_cells(dev, oracle, n):
    from paragram_b200 import workloads as W

    pts, w = W.power_uniform(n, seed=7)
    exp = oracle.diagram(pts, w)
    got = _gpu(dev, pts, w)
    _assert_same(got, exp, f"power{n}")
    if n >= 50_000:
        assert (exp[2] == 3).sum() > 0  # the configuration has empty cells


def test_power_heavy_weights(dev, oracle):
    rng = np.random.default_rng(5)
    pts = rng.random((3000, 3)).astype(np.float32)
    w = (rng.random(3000) * 0.02).astype(np.float32)
    _assert_same(_gpu(dev, pts, w), oracle.diagram(pts, w), "heavy")


def test_clustered(dev, oracle):
    from paragram_b200 import workloads as W

    pts = W.clustered(100_000, seed=4)
    _assert_same(_gpu(dev, pts), oracle.diagram(pts), "clustered100k")


def test_surface_clouds(dev, oracle):
    from paragram_b200 import workloads as W

    for k, c in enumerate(W.surface_clouds(num_clouds=4, seed=9, size_scale=0.05)):
        _assert_same(_gpu(dev, c), oracle.diagram(c), f"cloud{k}")


def test_jittered_lattice_power(dev, oracle):
    from paragram_b200 import workloads as W

    pts, w = W.jittered_lattice(24, seed=1)
    _assert_same(_gpu(dev, pts, w), oracle.diagram(pts, w), "lattice24")


@pytest.mark.parametrize("kind", ["lattice", "duplicates", "coplanar", "collinear"])
def test_degenerate(dev, oracle, kind):
    rng = np.random.default_rng(11)
    if kind == "lattice":
        pts = np.array(list(itertools.product(np.linspace(0.1, 0.9, 6), repeat=3)), np.float32)
    elif kind == "duplicates":
        p = rng.random((200, 3)).astype(np.float32)
        pts = np.concatenate([p, p[:50]])
    elif kind == "coplanar":
        pts = rng.random((500, 3)).astype(np.float32)
        pts[:, 0] = 0.5
    else:
        pts = np.stack([np.sort(rng.random(50)), np.full(50, 0.5), np.full(50, 0.5)], 1).astype(np.float32)
    _assert_same(_gpu(dev, pts), oracle.diagram(pts), kind)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden_fixtures(dev, path):
    f = np.load(path)
    w = f["weights"] if "weights" in f.files else None
    _assert_same(_gpu(dev, f["points"], w), (f["adjacency"], f["offsets"], f["status"]), os.path.basename(path))


def test_results_independent_of_knobs(dev):
    """knn, leaf_size and the chunk count are performance knobs only."""
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    pts, w = W.power_uniform(30_000, seed=2)
    t = torch.from_numpy(pts).to(dev)
    tw = torch.from_numpy(w).to(dev)
    base = [x.cpu() for x in pc.build_with_stats(t, tw)[0]]
    for kw in [dict(knn=0), dict(leaf_size=4), dict(leaf_size=32), dict(num_chunks=3), dict(knn=0, leaf_size=7)]:
        got = [x.cpu() for x in pc.build_with_stats(t, tw, **kw)[0]]
        assert all(torch.equal(a, b) for a, b in zip(base, got)), kw


def test_initial_guesses_do_not_change_results(dev, oracle):
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    pts = W.uniform(5000, seed=8)
    exp = oracle.diagram(pts)
    t = torch.from_numpy(pts).to(dev)
    d = pg.voronoi_diagram(t)
    # the true neighbours, random ids with duplicates and invalid ids, and empty lists
    rng = np.random.default_rng(0)
    rnd = rng.integers(-3, 5003, size=5000 * 6).astype(np.int32)
    for guesses, offs in [(d.adjacency, d.offsets),
                          (torch.from_numpy(rnd).to(dev), torch.arange(0, 5000 * 6 + 1, 6, dtype=torch.int32,
                                                                       device=dev)),
                          (torch.zeros(0, dtype=torch.int32, device=dev), torch.zeros(5001, dtype=torch.int32,
                                                                                      device=dev))]:
        g = pg.voronoi_diagram(t, initial_guesses=guesses, initial_guesses_offsets=offs)
        _assert_same((g.adjacency.cpu().numpy(), g.offsets.cpu().numpy(), g.status.cpu().numpy()), exp, "guesses")


def test_full_size_properties(dev):
    """5M clustered Voronoi: symmetric, sorted, no self loops, consistent offsets."""
    from paragram_b200 import workloads as W

    pts = W.clustered(5_000_000, seed=0)
    adj, off, st = _gpu(dev, pts)
    n = len(pts)
    assert off[0] == 0 and off[-1] == adj.size and (np.diff(off) >= 0).all()
    assert set(np.unique(st).tolist()) <= {0, 2}
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    assert (adj != rows).all()
    # sorted rows: within a row the sequence increases
    inc = np.diff(adj.astype(np.int64))
    same_row = np.diff(rows) == 0
    assert (inc[same_row] > 0).all()
    # symmetric: the edge set equals its transpose
    key = rows * n + adj
    tkey = adj.astype(np.int64) * n + rows
    assert np.array_equal(np.sort(key), np.sort(tkey))
    deg = np.diff(off)
    assert 14.0 < deg.mean() < 17.0


def test_low_level_errors(dev):
    import paragram_b200.cuda as pc

    pts = torch.rand(10, 3, device=dev)
    with pytest.raises(RuntimeError, match="weights must have 1 dimension"):
        pc.build_laguerre_voronoi_ultra(pts, torch.rand(10, device=dev))
    with pytest.raises(RuntimeError, match="points must be of type float"):
        pc.build_voronoi_ultra(pts.double())
    with pytest.raises(RuntimeError, match="leaf_size"):
        pc.build_voronoi_ultra(pts, leaf_size=99)


def test_empty_input(dev):
    import paragram_b200 as pg

    d = pg.voronoi_diagram(torch.zeros(0, 3, device=dev))
    assert d.adjacency.numel() == 0 and d.offsets.tolist() == [0] and d.status.numel() == 0


def _lattice_block(m, lo, k, seed):
    """k^3 points of the jittered m^3 lattice (spacing 1/m, jitter +-1e-4 spacing) and its weights."""
    rng = np.random.default_rng(seed)
    s = 1.0 / m
    idx = np.arange(lo, lo + k, dtype=np.float64)
    g = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), -1).reshape(-1, 3)
    pts = ((g + 0.5) * s + rng.uniform(-1e-4 * s, 1e-4 * s, size=g.shape)).astype(np.float32)
    w = (rng.random(len(g)) * 0.1 * s * s).astype(np.float32)
    return pts, w


def test_lattice_hull_cells_stay_local(dev, oracle):
    """Hull cells of a 1/310-spaced jittered lattice are prisms reaching the box 1.0 away, with
    nearly dependent plane triples along their edges. Exact results, and the traversal of those
    cells stays local (their empty spheres are not inflated by FP32 vertex error)."""
    import paragram_b200.cuda as pc

    pts, w = _lattice_block(310, 120, 24, seed=11)
    for wt in (w, None):
        t = torch.from_numpy(pts).to(dev)
        tw = None if wt is None else torch.from_numpy(wt).to(dev)
        (a, o, s), st = pc.build_with_stats(t, tw, diagnostics=True)
        _assert_same((a.cpu().numpy(), o.cpu().numpy(), s.cpu().numpy()), oracle.diagram(pts, wt), "lattice block")
        work = st["work"].cpu().numpy()
        g = np.round(pts * 310 - 0.5).astype(np.int64) - 120
        hull = (np.minimum(g, 23 - g).min(1) == 0)
        assert hull.sum() > 0
        assert work[hull, 0].mean() < 400, work[hull].mean(0)   # BVH nodes per hull cell
        assert work[:, 3].max() < 256                          # node queue never near its capacity


def test_diagnostics(dev, oracle):
    """Per-cell certified radius and work counters: a face of the final cell lies within the
    radius, so every neighbour q satisfies |q - s| / 2 <= R for Voronoi."""
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    pts = W.clustered(30000, seed=8)
    (a, o, s), st = pc.build_with_stats(torch.from_numpy(pts).to(dev), diagnostics=True)
    a, o = a.cpu().numpy(), o.cpu().numpy()
    R = st["radius"].cpu().numpy()
    work = st["work"].cpu().numpy()
    assert R.shape == (len(pts),) and work.shape == (len(pts), 4)
    assert (R > 0).all()
    src = np.repeat(np.arange(len(pts)), np.diff(o))
    half = 0.5 * np.linalg.norm(pts[a].astype(np.float64) - pts[src], axis=1)
    assert (half <= R[src].astype(np.float64) * (1 + 1e-5)).all()
    assert (work >= 0).all() and (work[:, 0] >= 1).all()
    assert (work[:, 2] >= np.diff(o)).all()  # every face neighbour was a tested candidate
    # deferred cells are counted twice in the totals (fast pass, then the 256-slot pass)
    assert int(work[:, 0].sum()) <= st["nodes"] and int(work[:, 1].sum()) <= st["leaves"]


@pytest.mark.parametrize("scale", [1.001, 0.5, 3.0, 0.0, -1.0, float("nan")])
def test_radius_hint_never_changes_results(dev, oracle, scale):
    """A search radius per cell (about right, too small, too large, absent or invalid) changes
    the work, never the diagram: the capped pass is certified, else an unbounded pass completes it."""
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    for pts, w in ((W.clustered(20000, seed=12), None), W.power_uniform(8000, seed=13)):
        t = torch.from_numpy(pts).to(dev)
        tw = None if w is None else torch.from_numpy(w).to(dev)
        (a, o, s), st = pc.build_with_stats(t, tw, diagnostics=True)
        hint = st["radius"] * scale
        (a2, o2, s2), st2 = pc.build_with_stats(t, tw, radius_hint=hint)
        assert torch.equal(a, a2) and torch.equal(o, o2) and torch.equal(s, s2)
        _assert_same((a2.cpu().numpy(), o2.cpu().numpy(), s2.cpu().numpy()), oracle.diagram(pts, w), f"hint x{scale}")
        if scale > 1.0:
            assert st2["hint_misses"] <= 0.01 * len(pts)
        if scale == 0.5:
            assert st2["hint_misses"] > 0.5 * len(pts)
        if not scale > 0.0:
            assert st2["hint_hits"] + st2["hint_misses"] == 0


def test_fp32_only_predicates(dev, oracle):
    """FP32-only side tests (the reference's arithmetic, no escalation): no FP64 or exact work,
    and on inputs in general position the same diagram as the exact path."""
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    for pts, w in ((W.uniform(20000, seed=21), None), W.power_uniform(20000, seed=22)):
        t = torch.from_numpy(pts).to(dev)
        tw = None if w is None else torch.from_numpy(w).to(dev)
        (a, o, s), st = pc.build_with_stats(t, tw, fp32_only=True)
        assert st["fp64_escalations"] == 0 and st["exact_escalations"] == 0
        _assert_same((a.cpu().numpy(), o.cpu().numpy(), s.cpu().numpy()), oracle.diagram(pts, w), "fp32 only")


@pytest.mark.parametrize("env", [{"PARAGRAM_NUM_CHUNKS": "4"}, {"PARAGRAM_MEM_FRAC": "0.06"},
                                 {"PARAGRAM_NUM_CHUNKS": "0", "PARAGRAM_MEM_FRAC": "2.0"}])
def test_chunk_environment(dev, monkeypatch, env):
    """The reference's chunk-plan environment (chunking.h:16-37) splits the cell pass into launches;
    the diagram is identical. PARAGRAM_MEM_FRAC outside (0.05, 0.95) is ignored, as in the reference."""
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    pts = W.clustered(40_000, seed=17)
    t = torch.from_numpy(pts).to(dev)
    base = [x.cpu() for x in pc.build_with_stats(t)[0]]
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    got = [x.cpu() for x in pc.build_with_stats(t, profile=True)[0]]
    assert all(torch.equal(a, b) for a, b in zip(base, got))
    chunks = pc.last_profile()["chunks"]
    if env.get("PARAGRAM_NUM_CHUNKS") == "4":
        assert chunks == 4


def test_search_radius_saves_candidates(dev, oracle):
    """What a search radius buys: with radii near the exact ones the first pass skips the far
    candidates of the first leaves (transient clips), the diagram unchanged."""
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    pts = W.clustered(200_000, seed=31)
    t = torch.from_numpy(pts).to(dev)
    (a, o, s), st = pc.build_with_stats(t, diagnostics=True)
    (a2, o2, s2), st2 = pc.build_with_stats(t, radius_hint=st["radius"] * 1.001)
    assert torch.equal(a, a2) and torch.equal(o, o2) and torch.equal(s, s2)
    assert st2["hint_misses"] == 0
    assert st2["candidates"] < 0.8 * st["candidates"], (st2["candidates"], st["candidates"])
    assert st2["clips"] < st["clips"]


def test_iterative_warm_start(dev, oracle):
    """Points that move a little between iterations, each iteration rebuilt with the previous
    iteration's diagram as initial guesses (plain, and with the learned search radius): every
    rebuild equals the cold build of the same points and the oracle, and the warm start saves
    traversal work (fewer BVH nodes and fewer clips per cell than the cold build)."""
    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import learned
    from paragram_b200 import workloads as W

    n = 200_000
    rng = np.random.default_rng(31)
    x = W.uniform(n, seed=31)
    step = 0.01 * (1.0 / n) ** (1.0 / 3.0)
    model = learned.train([learned.collect(torch.from_numpy(W.uniform(n, seed=32)).to(dev))], epochs=2, batch=8192)
    model.calibrate(learned.collect(torch.from_numpy(W.uniform(n, seed=33)).to(dev)), quantile=0.98)
    prev = pg.voronoi_diagram(torch.from_numpy(x).to(dev))
    for it in range(3):
        x = (x + step * rng.standard_normal(x.shape)).astype(np.float32)
        t = torch.from_numpy(x).to(dev)
        (a0, o0, s0), cold = pc.build_with_stats(t)
        (a1, o1, s1), warm = pc.build_with_stats(t, initial_guesses=prev.adjacency,
                                                 initial_guesses_offsets=prev.offsets)
        assert torch.equal(a1, a0) and torch.equal(o1, o0) and torch.equal(s1, s0), it
        assert warm["nodes"] < cold["nodes"] and warm["clips"] < cold["clips"], (it, warm, cold)
        d = learned.voronoi_diagram(t, model, initial_guesses=prev.adjacency, initial_guesses_offsets=prev.offsets)
        assert torch.equal(d.adjacency, a0) and torch.equal(d.offsets, o0) and torch.equal(d.status, s0), it
        if it == 0:
            _assert_same((a1.cpu().numpy(), o1.cpu().numpy(), s1.cpu().numpy()), oracle.diagram(x), "warm start")
        prev = pg.Diagram(adjacency=a1, offsets=o1, status=s1)
