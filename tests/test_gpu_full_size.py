"""Full-size parity: every benchmark configuration at its stated size, GPU against the oracle.

Bar: bit-identical sorted rows, offsets and statuses (the exact predicates).
The FP32-only predicate mode (the reference's arithmetic) is compared too; its
disagreements with the exact diagram are counted and bounded, since an FP32
decision inside its rounding error may go either way.

Sizes: 1M uniform power points, 5M clustered points (plain and learned search
radius), the 256 surface clouds of the batched configuration (one CUDA-graph
build), and the full 310^3 jittered power lattice. The oracle runs with every
host thread; its time and thread count are printed.
"""

import time

import numpy as np
import pytest
import torch
from _helpers import diff_cells as _diff_cells

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _np(d):
    return d.adjacency.cpu().numpy(), d.offsets.cpu().numpy(), d.status.cpu().numpy()


def _oracle(oracle, pts, w=None):
    t0 = time.perf_counter()
    c = oracle.cells(pts, w)
    adj, off = oracle.symmetrize(len(pts), c.row_offsets, c.rows)
    print(f"oracle: {len(pts)} cells in {time.perf_counter() - t0:.1f} s on {c.threads} threads")
    return adj, off, c.status


def test_power_1m_both_predicate_modes(dev, oracle):
    """Power diagram of 1M uniform points (weights up to 0.25 s^2; some cells are empty)."""
    import paragram_b200 as pg
    import paragram_b200.cuda as pc
    from paragram_b200 import workloads as W

    pts, w = W.power_uniform(1_000_000, seed=0)
    exp = _oracle(oracle, pts, w)
    assert (exp[2] == 3).sum() > 0
    t, tw = torch.from_numpy(pts).to(dev), torch.from_numpy(w).to(dev)
    got = _np(pg.power_diagram(t, tw))
    bad = _diff_cells(got, exp)
    assert bad.size == 0, f"{bad.size} cells differ, first {bad[:5].tolist()}"
    (a, o, s), st = pc.build_with_stats(t, tw, fp32_only=True)
    bad32 = _diff_cells((a.cpu().numpy(), o.cpu().numpy(), s.cpu().numpy()), exp)
    print(f"FP32-only predicates: {bad32.size} of {len(pts)} cells differ from the exact diagram")
    assert st["fp64_escalations"] == 0
    assert bad32.size <= 50


def test_clustered_5m_plain_and_learned(dev, oracle):
    """5M clustered Voronoi points, plain and with a learned search radius trained on other seeds."""
    import paragram_b200 as pg
    from paragram_b200 import learned
    from paragram_b200 import workloads as W

    pts = W.clustered(5_000_000, seed=0)
    exp = _oracle(oracle, pts)
    t = torch.from_numpy(pts).to(dev)
    plain = _np(pg.voronoi_diagram(t))
    bad = _diff_cells(plain, exp)
    assert bad.size == 0, f"plain: {bad.size} cells differ, first {bad[:5].tolist()}"
    data = [learned.collect(torch.from_numpy(W.clustered(300_000, seed=1000 + k)).to(dev)) for k in range(2)]
    model = learned.train(data, epochs=3, batch=8192)
    model.calibrate(data[0], quantile=0.98)
    got = _np(learned.voronoi_diagram(t, model))
    bad = _diff_cells(got, exp)
    assert bad.size == 0, f"learned: {bad.size} cells differ, first {bad[:5].tolist()}"


def test_surface_batch_256(dev, oracle):
    """The 256 uneven surface clouds, built as one batch from a captured CUDA graph."""
    from paragram_b200 import batch
    from paragram_b200 import workloads as W

    clouds = W.surface_clouds(num_clouds=256, seed=0)
    tens = [torch.from_numpy(c).to(dev) for c in clouds]
    batch.build_batch(tens, graph=True)  # capture
    out = batch.build_batch(tens, graph=True)  # replay
    t0 = time.perf_counter()
    total_bad = 0
    for k, (c, d) in enumerate(zip(clouds, out)):
        adj, off = None, None
        cc = oracle.cells(c)
        adj, off = oracle.symmetrize(len(c), cc.row_offsets, cc.rows)
        bad = _diff_cells(_np(d), (adj, off, cc.status))
        total_bad += bad.size
        assert bad.size == 0, f"cloud {k}: {bad.size} cells differ, first {bad[:5].tolist()}"
    print(f"oracle: {sum(len(c) for c in clouds)} cells of 256 clouds in {time.perf_counter() - t0:.1f} s")
    assert total_bad == 0


def test_lattice_310_power(dev, oracle):
    """The full jittered 310^3 power lattice (29.8M points, near-cospherical vertices everywhere)."""
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    pts, w = W.jittered_lattice(310, seed=0)
    t, tw = torch.from_numpy(pts).to(dev), torch.from_numpy(w).to(dev)
    got = _np(pg.power_diagram(t, tw))
    del t, tw
    torch.cuda.empty_cache()
    exp = _oracle(oracle, pts, w)
    bad = _diff_cells(got, exp)
    assert bad.size == 0, f"{bad.size} cells differ, first {bad[:5].tolist()}"


def test_max_size_uniform(dev, oracle):
    """The largest input the LBVH's leaf references allow, N = 2^26 - 1 uniform points (1.04G
    directed entries): the build completes with every status 0 or 2, every row sorted and the CSR
    symmetric (all entries, checked on the device), and the first 10,000 cells equal the oracle's
    exact rows (the exact Voronoi diagram of points in general position has no empty cell and its
    directed rows are already symmetric)."""
    import paragram_b200 as pg
    from paragram_b200 import workloads as W

    n = (1 << 26) - 1
    pts = W.uniform(n, seed=81)
    d = pg.voronoi_diagram(torch.from_numpy(pts).to(dev))
    adj, off, st = d.adjacency, d.offsets.long(), d.status
    e = adj.numel()
    assert int(off[-1]) == e and e > 14 * n
    assert bool(((st == 0) | (st == 2)).all())
    deg = off[1:] - off[:-1]
    rows = torch.repeat_interleave(torch.arange(n, device=dev), deg)
    # sorted rows: a row's entries increase; (row, column) keys are then globally sorted
    keys = rows * n + adj.long()
    del rows
    assert bool((keys[1:] > keys[:-1]).all())
    # symmetric: every (u, v) has its (v, u)
    cols = adj.long()
    rkeys = cols * n + torch.repeat_interleave(torch.arange(n, device=dev), deg)
    del cols
    pos = torch.searchsorted(keys, rkeys).clamp_max(e - 1)
    assert bool((keys[pos] == rkeys).all())
    del keys, rkeys, pos
    m = 10_000
    t0 = time.perf_counter()
    c = oracle.cells(pts, None, begin=0, end=m)
    print(f"oracle: {m} of {n} cells (kd-tree over all points) in {time.perf_counter() - t0:.1f} s")
    got_off = off[: m + 1].cpu().numpy()
    got = adj[: int(got_off[-1])].cpu().numpy()
    exp_off = c.row_offsets.astype(np.int64)
    rid = np.repeat(np.arange(m), np.diff(exp_off))
    exp = c.rows.astype(np.int64)[np.lexsort((c.rows, rid))]
    assert np.array_equal(got_off, exp_off)
    assert np.array_equal(got.astype(np.int64), exp)
    assert np.array_equal(st[:m].cpu().numpy(), c.status)
